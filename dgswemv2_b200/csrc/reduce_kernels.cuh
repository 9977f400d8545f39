// FP64 reductions over elements and state-layout permutations.
//
// L2 error: Simulation::ComputeL2Residual (source/simulation/serial/simulation.hpp:85-93) with
// Element::ComputeResidualL2 (source/geometry/element.hpp:549-592): per element sum over the three
// variables of int (true_q(t, x) - q_h)^2 dA with a degree-20 rule, |J| outside the quadrature sum.
// The rule here is the collapsed Gauss-Legendre x Gauss-Jacobi(1,0) product rule of degree 20
// (121 points), exact to the same polynomial degree as the reference's 79-point Dunavant rule.
// Mass: sum_e int_e (ze_h + b_h) dA = sum_e 2 |J| (ze_0 + b_0) (phi_0 = 1, master area 2).
// Each block reduces its elements in a fixed tree order and writes one partial; the host adds the
// partials in block order, so the result does not depend on scheduling.
#ifndef DGSW_REDUCE_KERNELS_CUH
#define DGSW_REDUCE_KERNELS_CUH

#include <cuda_runtime.h>

#include "function_sets.h"

namespace dgsw {

constexpr int L2_NPT = 121;
constexpr int RED_BLOCK = 256;

struct L2Rule {
    double w[L2_NPT];
    double psi[3][L2_NPT];
    double phi[2][6 * L2_NPT];  // [p-1][dof][pt]
};

template <typename Real>
struct ReduceArgs {
    const double* q;   // FP64 state (both precisions)
    const Real* bath;
    const int* enodes;
    const double2* xy;
    int ne, ne_pad;
    double t;
    int fn_set;
    double fn_params[16];
    double* partial;
    int npartial;
    const L2Rule* rule;  // device copy of the degree-20 rule and basis values
};

inline int64_t reduction_partials(int64_t ne) { return (ne + RED_BLOCK - 1) / RED_BLOCK; }

__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = RED_BLOCK / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    return sh[0];
}

template <int ND, typename Real>
__global__ void __launch_bounds__(RED_BLOCK) l2_error_kernel(const ReduceArgs<Real> R) {
    __shared__ double sh[RED_BLOCK];
    const int e = blockIdx.x * RED_BLOCK + threadIdx.x;
    double val = 0.0;
    if (e < R.ne) {
        const size_t P = (size_t)R.ne_pad;
        const int n0 = R.enodes[e], n1 = R.enodes[P + e], n2 = R.enodes[2 * P + e];
        const double2 X0 = R.xy[n0], X1 = R.xy[n1], X2 = R.xy[n2];
        const double J00 = (X1.x - X0.x) / 2.0, J01 = (X2.x - X0.x) / 2.0;
        const double J10 = (X1.y - X0.y) / 2.0, J11 = (X2.y - X0.y) / 2.0;
        const double aJ = fabs(J00 * J11 - J10 * J01);
        double q[3][ND];
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < ND; ++k) q[v][k] = (double)R.q[(v * ND + k) * P + e];
        const L2Rule& RL = *R.rule;
        const double* phi = RL.phi[ND == 3 ? 0 : 1];
        double l2[3] = {0.0, 0.0, 0.0};
        for (int gp = 0; gp < L2_NPT; ++gp) {
            const double x = X0.x * RL.psi[0][gp] + X1.x * RL.psi[1][gp] + X2.x * RL.psi[2][gp];
            const double y = X0.y * RL.psi[0][gp] + X1.y * RL.psi[1][gp] + X2.y * RL.psi[2][gp];
            const dgsw_fn3 f = dgsw_fn_true(R.fn_set, R.fn_params, R.t, x, y);
            const double tv[3] = {f.ze, f.qx, f.qy};
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                double u = 0.0;
#pragma unroll
                for (int k = 0; k < ND; ++k) u += q[v][k] * phi[k * L2_NPT + gp];
                const double dd = tv[v] - u;
                l2[v] += (dd * dd) * RL.w[gp];
            }
        }
        val = l2[0] * aJ + l2[1] * aJ + l2[2] * aJ;
    }
    const double s = block_sum(val, sh);
    if (threadIdx.x == 0) R.partial[blockIdx.x] = s;
}

template <int ND, typename Real>
__global__ void __launch_bounds__(RED_BLOCK) mass_kernel(const ReduceArgs<Real> R) {
    __shared__ double sh[RED_BLOCK];
    const int e = blockIdx.x * RED_BLOCK + threadIdx.x;
    double val = 0.0;
    if (e < R.ne) {
        const size_t P = (size_t)R.ne_pad;
        const double2 X0 = R.xy[R.enodes[e]], X1 = R.xy[R.enodes[P + e]], X2 = R.xy[R.enodes[2 * P + e]];
        const double det = (X1.x - X0.x) / 2.0 * ((X2.y - X0.y) / 2.0) - (X1.y - X0.y) / 2.0 * ((X2.x - X0.x) / 2.0);
        val = 2.0 * fabs(det) * ((double)R.q[e] + (double)R.bath[e]);
    }
    const double s = block_sum(val, sh);
    if (threadIdx.x == 0) R.partial[blockIdx.x] = s;
}

template <typename Real>
cudaError_t launch_reduction(const ReduceArgs<Real>& R, int p, int what, cudaStream_t st) {
    const int blocks = (R.ne + RED_BLOCK - 1) / RED_BLOCK;
    if (blocks > R.npartial) return cudaErrorInvalidValue;
    if (what == 0) {
        if (p == 1)
            l2_error_kernel<3, Real><<<blocks, RED_BLOCK, 0, st>>>(R);
        else
            l2_error_kernel<6, Real><<<blocks, RED_BLOCK, 0, st>>>(R);
    } else {
        if (p == 1)
            mass_kernel<3, Real><<<blocks, RED_BLOCK, 0, st>>>(R);
        else
            mass_kernel<6, Real><<<blocks, RED_BLOCK, 0, st>>>(R);
    }
    return cudaGetLastError();
}

// element-major [ref][comp] <-> component-major [comp][ne_pad] in device order, with a precision
// conversion (the host-facing state is FP64 in every precision)
template <typename Src, typename Dst>
__global__ void permute_in_kernel(const Src* __restrict__ src, Dst* __restrict__ dst, const int* __restrict__ ref_of_dev,
                                  int ne, int ne_pad, int ncomp) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ne) return;
    const int r = ref_of_dev[d];
    for (int c = 0; c < ncomp; ++c) dst[c * ne_pad + d] = (Dst)src[(size_t)r * ncomp + c];
}

template <typename Src, typename Dst>
__global__ void permute_out_kernel(const Src* __restrict__ src, Dst* __restrict__ dst,
                                   const int* __restrict__ ref_of_dev, int ne, int ne_pad, int ncomp) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ne) return;
    const int r = ref_of_dev[d];
    for (int c = 0; c < ncomp; ++c) dst[(size_t)r * ncomp + c] = (Dst)src[c * ne_pad + d];
}

template <typename Src, typename Dst>
cudaError_t launch_permute_in(const Src* src, Dst* dst, const int* ref_of_dev, int ne, int ne_pad, int ncomp,
                              cudaStream_t s) {
    permute_in_kernel<Src, Dst><<<(ne + 255) / 256, 256, 0, s>>>(src, dst, ref_of_dev, ne, ne_pad, ncomp);
    return cudaGetLastError();
}

template <typename Src, typename Dst>
cudaError_t launch_permute_out(const Src* src, Dst* dst, const int* ref_of_dev, int ne, int ne_pad, int ncomp,
                               cudaStream_t s) {
    permute_out_kernel<Src, Dst><<<(ne + 255) / 256, 256, 0, s>>>(src, dst, ref_of_dev, ne, ne_pad, ncomp);
    return cudaGetLastError();
}

}  // namespace dgsw

#endif
