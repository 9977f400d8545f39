// Stage-kernel instantiations for polynomial order 1, FP32 arithmetic, the autotuner's alternative register
// budget (compiled as a separate unit).
#include "stage_kernel.cuh"

namespace dgsw {
cudaError_t launch_stage_p1_f32_occ(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s) {
    return launch_stage_dispatch<1, float, 1>(A, tile, ntiles, max_halo, max_edges, mode, s);
}
}  // namespace dgsw
