// Stage-kernel instantiations for polynomial order 1, FP32 arithmetic with the intermediate stage states
// kept as FP32 increments from a carried state held as two FP32 parts (both register budgets; compiled as a
// separate unit).
#include "stage_kernel.cuh"

namespace dgsw {
cudaError_t launch_stage_p1_f32_split(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                      int mode, cudaStream_t s) {
    if (mode & STAGE_MODE_OCC) return launch_stage_split_dispatch<1, 1>(A, tile, ntiles, max_halo, max_edges, mode, s);
    return launch_stage_split_dispatch<1, 0>(A, tile, ntiles, max_halo, max_edges, mode, s);
}
}  // namespace dgsw
