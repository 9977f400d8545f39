// Stage-kernel instantiations for polynomial order 2, FP64 arithmetic, the autotuner's alternative register
// budget (compiled as a separate unit).
#include "stage_kernel.cuh"

namespace dgsw {
cudaError_t launch_stage_p2_f64_occ(const StageArgs<double>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s) {
    return launch_stage_dispatch<2, double, 1>(A, tile, ntiles, max_halo, max_edges, mode, s);
}
}  // namespace dgsw
