// Cooperative packed sweep kernels for one direction (see l1gs_coop_kernel.cuh).
#include "l1gs_coop_kernel.cuh"

namespace hscoop {
template int launch_dir<0>(int sdt, int io, int tpp, int m, const Params& p, LaunchCache* lc, cudaStream_t st);
}  // namespace hscoop
