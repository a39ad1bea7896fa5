// Dispatch of the cooperative packed sweep (kernels: l1gs_coop_kernel.cuh,
// compiled per direction in l1gs_coop_fwd.cu / _bwd.cu / _sym.cu).
#include "l1gs_coop.cuh"

namespace hscoop {

template <int SWEEP>
int launch_dir(int sdt, int io, int tpp, int m, const Params& p, LaunchCache* lc, cudaStream_t st);

bool supported(int ps, int tpp, int m) {
    // (8 lanes: the blocked kernel, partsizes that are multiples of 8)
    const bool pair = (tpp == 4 || tpp == 16 || tpp == 32) && (m == 4 || m == 8 || m == 16);
    if (!pair) return false;
    return ps == tpp * m || tpp == 16 || tpp == 32;
}

int launch(int sdt, int io, int sweep, int tpp, int m, const Params& p, LaunchCache* lc, cudaStream_t st) {
    if (p.gend <= p.gbeg) return HS_OK;
    if (p.blk) return launch_blk(sdt, io, sweep, p, lc, st);
    switch (sweep) {
        case HS_SWEEP_FORWARD: return launch_dir<0>(sdt, io, tpp, m, p, lc, st);
        case HS_SWEEP_BACKWARD: return launch_dir<1>(sdt, io, tpp, m, p, lc, st);
        default: return launch_dir<2>(sdt, io, tpp, m, p, lc, st);
    }
}

}  // namespace hscoop
