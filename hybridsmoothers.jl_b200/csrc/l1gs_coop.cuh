// Cooperative packed L1 Gauss-Seidel sweep: TPP lanes per partition.
//
// Reference: the packed sweep of src/l1_gauss_seidel.jl (:1068-1095 with the
// accumulations :1547-1585) computes, per partition, y_i = (y_i - acc_i)/D_i
// with acc_i = sum_j a_ij y_j over the partition's strict triangle, rows
// ascending (forward) or descending (backward), one thread per partition.
// With few partitions (large partsizes) that leaves most of the GPU idle, so
// here a partition is shared by TPP lanes of a warp (G = 32/TPP partitions per
// warp, a "group"), each lane owning rows r, r+TPP, r+2 TPP, ...  The sweep is
// right-looking: once row j is solved, its value is broadcast to the
// partition's lanes by a shuffle and every remaining row adds a_ij * y_j to
// its accumulator.  Forward, a row therefore receives its terms in ascending j
// -- the reference's order, so the forward sweep is bit-identical to it.
// Backward, terms arrive in descending j (the reference sums ascending), so
// backward and symmetric results agree with the reference to rounding
// (relative 1e-12 is the contract), not bitwise.
//
// Coefficients are stored column by column in the order the sweep consumes
// them ("coop" layout).  A group's stream holds, per direction, ps column
// blocks; block t has G * len_t entries, len_t = ps-1-t, entry e of partition
// g at e*G + g:
//   lower (forward),  block t = column j = t:      entry e is a_{j+1+e, j}
//   upper (backward), block t = column j = ps-1-t: entry e is a_{e, j}
// so every block is one contiguous run and the lanes of a warp read
// consecutive addresses.  A symmetric handle keeps the upper blocks after the
// lower ones in the same group stream.  Each warp pulls its groups' streams
// through a ring of shared-memory chunks filled by 1D bulk copies
// (cp.async.bulk, no multicast), STAGES-1 chunks ahead, across group
// boundaries.  Padding (the missing rows of a short last partition, the
// partitions that fill the last group) holds zeros and D_Dl1 = 1.
#pragma once

#include <algorithm>
#include <cstdlib>

#include "hs_common.cuh"

namespace hscoop {

// Blocked variant ("blk"): B = 8 lanes per partition, G = 4 partitions per
// warp, the partition (padded to psb, a multiple of 8, with zero rows and
// columns) cut into 8 x 8 tiles.
// The sweep is left-looking by row block: row block I first adds the
// off-diagonal tiles (I, J) of the blocks solved before it -- a dense
// product with y of those blocks, lanes = rows, no dependence between
// steps -- and then solves its diagonal tile, where the solved row's value is
// broadcast to the block's lanes by a shuffle.  Forward, row i adds its terms
// in ascending j (tiles J = 0, 1, ... then the diagonal tile's columns), the
// reference's order, so forward sweeps are bit-identical; backward and
// symmetric sweeps agree to rounding.  Stream order per direction and group:
//   lower: for I = 0 .. nb-1: tiles (I, 0 .. I-1), then diagonal tile I
//   upper: for I = nb-1 .. 0: tiles (I, I+1 .. nb-1), then diagonal tile I
// An off-diagonal warp tile (the G partitions' tiles) is 32 x 8 entries,
// [column / V][lane][column % V] with lane = g * 8 + row and V = 16 bytes /
// element size, so a lane reads V columns of its row with one 16-byte load;
// a diagonal warp tile keeps only its strict triangle, column by column in
// the order of the solve (lower: columns 0..6, rows below; upper: columns
// 7..1, rows above), partitions side by side inside a column.
constexpr int kBlkB = 8;

// Entries of direction blocks 0..t-1: G * sum_{u<t} (ps-1-u).
__host__ __device__ __forceinline__ int64_t colbase(int64_t ps, int64_t G, int64_t t) {
    return G * (t * (ps - 1) - t * (t - 1) / 2);
}

struct Layout {
    int32_t ps = 0, G = 0;
    int32_t blk = 0, V = 0;  // blocked variant; elements per 16 bytes
    int32_t psb = 0;         // blocked: ps rounded up to a multiple of 8 (rows past ps are padding)
    int64_t Ld = 0;          // entries per direction per group: G*ps*(ps-1)/2
    int64_t Lg = 0;          // entries of one group stream (Ld, or 2*Ld for both directions)
    int64_t Lgp = 0;         // group stride in the buffer: Lg rounded up to 128 bytes
    int64_t upper_off = 0;   // first upper entry inside a group stream (0, or Ld)
};

inline bool blk_ok(int ps, int tpp) { return tpp == kBlkB && ps >= kBlkB; }
inline int blk_psb(int ps) { return (ps + kBlkB - 1) / kBlkB * kBlkB; }
// Stream bytes of the padded blocked layout over the reference's triangles.
inline double blk_padding(int ps) {
    const double b = blk_psb(ps);
    return ps > 1 ? b * (b - 1) / ((double)ps * (ps - 1)) : 1e9;
}

inline Layout make_layout(int ps, int tpp, bool lower, bool upper, size_t es) {
    Layout L;
    L.ps = ps;
    L.G = 32 / tpp;
    L.blk = blk_ok(ps, tpp) ? 1 : 0;
    L.psb = L.blk ? blk_psb(ps) : ps;
    L.V = (int32_t)(16 / es);
    L.Ld = (int64_t)L.G * L.psb * (L.psb - 1) / 2;
    L.Lg = (lower && upper) ? 2 * L.Ld : L.Ld;
    const int64_t q = 128 / (int64_t)es;
    L.Lgp = (L.Lg + q - 1) / q * q;
    L.upper_off = lower ? L.Ld : 0;
    return L;
}

// Position of a_{li,lj} (local row/column of partition k) in the stream.
__host__ __device__ __forceinline__ int64_t lower_idx(const Layout& L, int64_t k, int64_t li, int64_t lj) {
    const int64_t q = k / L.G, g = k - q * L.G;
    if (L.blk) {
        constexpr int64_t B = kBlkB, TILE = 32 * B;
        const int64_t G = L.G, V = L.V, DG = G * B * (B - 1) / 2;
        const int64_t I = li / B, ii = li - I * B, J = lj / B, jj = lj - J * B;
        const int64_t rs = TILE * (I * (I - 1) / 2) + I * DG;   // row block I's first entry
        const int64_t off = J < I ? rs + J * TILE + (jj / V) * 32 * V + (g * B + ii) * V + jj % V
                                  : rs + I * TILE + G * (jj * (B - 1) - jj * (jj - 1) / 2) + g * (B - 1 - jj) +
                                        (ii - jj - 1);
        return q * L.Lgp + off;
    }
    return q * L.Lgp + colbase(L.ps, L.G, lj) + (li - lj - 1) * L.G + g;
}
__host__ __device__ __forceinline__ int64_t upper_idx(const Layout& L, int64_t k, int64_t li, int64_t lj) {
    const int64_t q = k / L.G, g = k - q * L.G;
    if (L.blk) {
        constexpr int64_t B = kBlkB, TILE = 32 * B;
        const int64_t G = L.G, V = L.V, DG = G * B * (B - 1) / 2;
        const int64_t I = li / B, ii = li - I * B, J = lj / B, jj = lj - J * B;
        const int64_t m = L.psb / B - 1 - I;                    // row blocks after I (consumed before it)
        const int64_t rs = TILE * (m * (m - 1) / 2) + m * DG;
        const int64_t off = J > I ? rs + (J - I - 1) * TILE + (jj / V) * 32 * V + (g * B + ii) * V + jj % V
                                  : rs + m * TILE + G * (B * (B - 1) / 2 - jj * (jj + 1) / 2) + g * jj + ii;
        return q * L.Lgp + L.upper_off + off;
    }
    return q * L.Lgp + L.upper_off + colbase(L.ps, L.G, L.ps - 1 - lj) + li * L.G + g;
}

// Per warp, shared memory holds a ring of `nst` chunks of 2^che_log2
// entries, then `ntail` more chunk slots that repeat the first `ntail` stages
// (every chunk copied into stage s < ntail is copied to stage nst + s as
// well), so a column block that starts anywhere in the ring is one linear
// run; then one mbarrier per stage, then y and D_Dl1 of the group's rows
// ([row][partition]).
struct Geometry {
    uint32_t che_log2 = 0;
    uint32_t nst = 0, ntail = 0;
    uint32_t bars_off = 0, ys_off = 0, ds_off = 0;   // byte offsets inside a warp's slice
    uint32_t warp_bytes = 0;
};

inline Geometry make_geometry(const Layout& L, size_t es) {
    Geometry g;
    if (L.blk) {   // the blocked kernel: a ring of 4 item slots (32 x 8 entries each), then y of the group
        g.ys_off = (uint32_t)(4 * 32 * kBlkB * es);
        g.warp_bytes = (uint32_t)((g.ys_off + (size_t)L.G * L.psb * es + 127) / 128 * 128);
        return g;
    }
    // Tuning overrides: HSB200_COOP_CHUNK = chunk bytes (1024, 2048 or 4096),
    // HSB200_COOP_AHEAD = chunks kept in flight beyond a column block (1..8).
    uint32_t chunk_bytes = 2048, ahead = 2;
    if (const char* env = getenv("HSB200_COOP_CHUNK")) {
        const int v = atoi(env);
        if (v == 1024 || v == 2048 || v == 4096) chunk_bytes = (uint32_t)v;
    }
    if (const char* env = getenv("HSB200_COOP_AHEAD")) {
        const int v = atoi(env);
        if (v >= 1 && v <= 8) ahead = (uint32_t)v;
    }
    const uint32_t che = (uint32_t)(chunk_bytes / es);
    while ((1u << g.che_log2) < che) ++g.che_log2;
    const int64_t maxcol = (int64_t)L.G * (L.ps - 1);        // entries of the longest column block
    g.ntail = (uint32_t)std::max<int64_t>(1, (maxcol + che - 1) / che);
    // A column block spans at most ntail + 1 chunks; keep `ahead` more in flight.
    g.nst = 4;
    while (g.nst < g.ntail + 1 + ahead) g.nst *= 2;
    const size_t ring = (size_t)(g.nst + g.ntail) * che * es;
    g.bars_off = (uint32_t)ring;
    g.ys_off = (uint32_t)((ring + 8 * g.nst + 15) / 16 * 16);
    const size_t rows = (size_t)L.G * L.ps * es;
    g.ds_off = (uint32_t)(g.ys_off + (rows + 15) / 16 * 16);
    g.warp_bytes = (uint32_t)((g.ds_off + rows + 127) / 128 * 128);
    return g;
}

struct Params {
    int32_t n, ps;
    int32_t blk;             // blocked layout and kernel
    int32_t gbeg, gend;      // groups [gbeg, gend) of this launch
    int32_t Lg;              // entries of one group stream
    int64_t Lgp;             // group stride in the buffer
    Geometry geo;
    const void* SC;          // group streams
    const void* D;           // D_Dl1 in natural row order
    const void* x;
    void* y;
    int32_t* err;
};

struct LaunchCache {
    const void* kern = nullptr;
    int wpb = 0, per_sm = 0;
};

// True when a kernel is instantiated for (partsize, lanes per partition,
// rows per lane).
bool supported(int ps, int tpp, int m);

// Launches the sweep for smoother type sdt (HS_F64/HS_F32) and vector type io.
int launch(int sdt, int io, int sweep, int tpp, int m, const Params& p, LaunchCache* lc, cudaStream_t st);
// The blocked kernel (l1gs_blk.cu).
int launch_blk(int sdt, int io, int sweep, const Params& p, LaunchCache* lc, cudaStream_t st);

// Rows per lane for (partsize, lanes per partition): the smallest power of
// two from 4 to 16 that covers ps, or 0.
constexpr int kMaxRowsPerLane = 16;
inline int rows_per_lane(int ps, int tpp) {
    const int need = (ps + tpp - 1) / tpp;
    for (int m = 4; m <= kMaxRowsPerLane; m *= 2)
        if (need <= m) return m;
    return 0;
}

}  // namespace hscoop
