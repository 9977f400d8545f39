// Arguments and launcher of the trouble-indicator kernels (trouble.cu).
#ifndef DGSW_TROUBLE_CUH
#define DGSW_TROUBLE_CUH

#include <cuda_runtime.h>

namespace dgsw {

template <typename Real>
struct TroubleArgs {
    const double* q;             // FP64 state [(var*ND+dof)][ne_pad]
    const Real* bath;            // bathymetry modes [3][ne_pad]
    const unsigned char* wet;    // wet flags of this state
    const int* nbr;              // [3][ne_pad] neighbour (device index) or -2 - boundary type
    const signed char* nbr_face; // [3][ne_pad] the neighbour's face across each face
    const int* enodes;           // [3][ne_pad]
    const double2* xy;
    const int* ref_of_dev;       // reference order = ascending element ID: the smaller is the "in" side
    double* I;                   // [ne] indicator (device order)
    unsigned char* flag;         // [ne] troubled before spreading
    int ne, ne_pad;
};

// indicator and initial flags into A.I / A.flag, then five neighbour layers of growth into `out`
template <typename Real>
cudaError_t launch_trouble(const TroubleArgs<Real>& A, int p, unsigned char* scratch, unsigned char* out,
                           cudaStream_t s);

}  // namespace dgsw

#endif
