// Output values for the VTK / VTU writers (write_VTK_data / write_VTU_data,
// problem_postprocessor/swe_post_write_vtk.hpp:5-95, swe_post_write_vtu.hpp:5-104, with the reference's
// N_DIV = 1): per element, u * phi_postprocessor_point at its three vertices and u * phi_postprocessor_cell
// at its centroid (Element::WritePointDataVTK / WriteCellDataVTK, element.hpp:513-533), for ze, qx, qy and
// the bathymetry, evaluated from the device state and scattered to ascending element-ID order.
#include <cuda_runtime.h>

#include "postprocess.cuh"

namespace dgsw {

template <typename Real>
__global__ void __launch_bounds__(256) postprocess_kernel(const PostArgs<Real> A) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= A.ne) return;
    const size_t P = (size_t)A.ne_pad;
    const int r = A.ref_of_dev[e];
    for (int pt = 0; pt < 4; ++pt) {
        double val[4];
        for (int v = 0; v < 3; ++v) {
            double s = 0.0;
            for (int k = 0; k < A.nd; ++k) s += A.q[(v * A.nd + k) * P + e] * A.phi[pt][k];
            val[v] = s;
        }
        double b = 0.0;
        for (int k = 0; k < 3; ++k) b += (double)A.bath[k * P + e] * A.phi[pt][k];
        val[3] = b;
        double* out = pt < 3 ? A.point + ((size_t)r * 3 + pt) * 4 : A.cell + (size_t)r * 4;
        for (int c = 0; c < 4; ++c) out[c] = val[c];
    }
    A.wet_out[r] = A.wet[e];
    A.went_dry_out[r] = A.went_dry ? A.went_dry[e] : 0;
}

template <typename Real>
cudaError_t launch_postprocess(const PostArgs<Real>& A, cudaStream_t s) {
    if (A.ne <= 0) return cudaSuccess;
    postprocess_kernel<Real><<<(unsigned)((A.ne + 255) / 256), 256, 0, s>>>(A);
    return cudaGetLastError();
}

template cudaError_t launch_postprocess<float>(const PostArgs<float>&, cudaStream_t);
template cudaError_t launch_postprocess<double>(const PostArgs<double>&, cudaStream_t);

}  // namespace dgsw
