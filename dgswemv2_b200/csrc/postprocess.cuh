// Arguments and launcher of the output evaluation kernel (postprocess.cu).
#ifndef DGSW_POSTPROCESS_CUH
#define DGSW_POSTPROCESS_CUH

#include <cuda_runtime.h>

namespace dgsw {

template <typename Real>
struct PostArgs {
    const double* q;                 // FP64 modal state [(var*ND+dof)][ne_pad]
    const Real* bath;                // bathymetry modes of the linear part [3][ne_pad]
    const unsigned char* wet;        // wet flags
    const unsigned char* went_dry;   // went-completely-dry flags, or null
    const int* ref_of_dev;           // output order = ascending element ID
    double phi[4][6];                // modes at vertices 0, 1, 2 and at the centroid
    double* point;                   // [ne][3][4] ze, qx, qy, bath at the vertices
    double* cell;                    // [ne][4] at the centroid
    unsigned char* wet_out;          // [ne]
    unsigned char* went_dry_out;     // [ne]
    int ne, ne_pad, nd;
};

template <typename Real>
cudaError_t launch_postprocess(const PostArgs<Real>& A, cudaStream_t s);

}  // namespace dgsw

#endif
