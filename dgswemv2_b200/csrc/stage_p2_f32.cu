// Stage-kernel instantiations for polynomial order 2, FP32 arithmetic, the default register budget
// (compiled as a separate unit).
#include "stage_kernel.cuh"

namespace dgsw {
cudaError_t launch_stage_p2_f32(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                int mode, cudaStream_t s) {
    return launch_stage_dispatch<2, float, 0>(A, tile, ntiles, max_halo, max_edges, mode, s);
}
}  // namespace dgsw
