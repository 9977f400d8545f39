// Arguments and launcher of the levee-interface flux pass (levee.cu).
#ifndef DGSW_LEVEE_CUH
#define DGSW_LEVEE_CUH

#include <cuda_runtime.h>

namespace dgsw {

constexpr int LEVEE_STRIDE_DEV = 17;  // nx, ny, H[3], C_sub[3], C_super[3], sp_in[3], sp_ex[3]

template <typename Real>
struct LeveeArgs {
    const double* q;           // this stage's FP64 state [(var*ND+dof)][ne_pad]
    const Real* bath;          // bathymetry modes [3][ne_pad]
    const unsigned char* wet;  // wet flags of this state
    const int4* lev;           // [n]: in element (device index), in face, ex element, ex face
    const double* ldat;        // [n][LEVEE_STRIDE_DEV]
    double* F;                 // [n][2][3][NG]: in-side flux at in Gauss point g, ex-side flux at the ex
                               // Gauss point NG-1-g (paired with g), stored at g
    int n, ne_pad;
    double g;
};

template <typename Real>
cudaError_t launch_levee(const LeveeArgs<Real>& A, int p, cudaStream_t s);

}  // namespace dgsw

#endif
