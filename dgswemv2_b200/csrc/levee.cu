// Levee interfaces (ISP::Levee::ComputeFlux, discretization_RKDG/interface_specializations/
// rkdg_swe_is_levee.hpp:64-175): one thread per levee interface computes, at each Gauss point, the two
// ghost states (reflective land states when both sides are below the crest plus the 0.01 m tolerance or
// within it of each other; otherwise the weir discharge from the higher side, subcritical
// C_sub h_low sqrt(2 g (h_high - h_low)) when the lower head exceeds 2/3 of the higher, else supercritical
// C_super (2/3 h_high) sqrt(g (2/3 h_high)), along the normal of the higher side, with gravity dropped
// on a dry receiving side) and the two LLF fluxes, in FP64, before the stage kernel runs; the stage
// kernel lifts them like any other edge flux. Levee interfaces are few, so this pass is tiny.
#include <cuda_runtime.h>

#include "levee.cuh"
#include "stage_kernel.cuh"

namespace dgsw {

template <int P, typename Real>
__device__ __forceinline__ void levee_trace(const LeveeArgs<Real>& A, int e, int f, double (&t)[4][MT<P>::NG]) {
    constexpr int ND = MT<P>::ND;
    const size_t Pp = (size_t)A.ne_pad;
    double q[3][ND], b[3];
#pragma unroll
    for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = A.q[c * Pp + e];
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] = (double)A.bath[k * Pp + e];
    if (f == 0)
        face_trace<P, 0, double>(q, b, t);
    else if (f == 1)
        face_trace<P, 1, double>(q, b, t);
    else
        face_trace<P, 2, double>(q, b, t);
}

// BC::Land::GetEX (rkdg_swe_bc_land.hpp:88-104): normal momentum mirrored, tangential kept
__device__ __forceinline__ void land_ghost(double nx, double ny, const double (&q)[3], double (&qe)[3]) {
    const double tx = -ny, ty = nx;
    const double qn = -(q[1] * nx + q[2] * ny);
    const double qt = q[1] * tx + q[2] * ty;
    qe[0] = q[0];
    qe[1] = qn * nx + qt * tx;
    qe[2] = qn * ny + qt * ty;
}

template <int P, typename Real>
__global__ void __launch_bounds__(128) levee_kernel(const LeveeArgs<Real> A) {
    constexpr int NG = MT<P>::NG;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= A.n) return;
    const int4 L = A.lev[l];
    const double* D = A.ldat + (size_t)l * LEVEE_STRIDE_DEV;
    const double nx = D[0], ny = D[1];
    const bool wet_in = A.wet[L.x] != 0, wet_ex = A.wet[L.z] != 0;
    double ti[4][NG], te[4][NG];
    levee_trace<P, Real>(A, L.x, L.y, ti);
    levee_trace<P, Real>(A, L.z, L.w, te);
    double* F = A.F + (size_t)l * 6 * NG;
    constexpr double tol = 0.01;  // H_tolerance
    double q_in_ex[3] = {0.0, 0.0, 0.0}, q_ex_ex[3] = {0.0, 0.0, 0.0};
    for (int g = 0; g < NG; ++g) {
        const int ge = NG - 1 - g;
        const double H = D[2 + g], Cs = D[2 + 3 + g], Cp = D[2 + 6 + g];
        const double qi[3] = {ti[0][g], ti[1][g], ti[2][g]};
        const double qe[3] = {te[0][ge], te[1][ge], te[2][ge]};
        double g_in = A.g, g_ex = A.g;
        const double hi = qi[0] - H, he = qe[0] - H;
        if ((hi <= tol && he <= tol) || fabs(hi - he) <= tol) {
            land_ghost(nx, ny, qi, q_in_ex);
            land_ghost(-nx, -ny, qe, q_ex_ex);
        } else if (hi > he) {  // overtopping from in to ex
            double qn;
            if (he > 2.0 * hi / 3.0)
                qn = Cs * he * sqrt(2.0 * A.g * (hi - he));
            else
                qn = Cp * (2.0 * hi / 3.0) * sqrt(A.g * (2.0 * hi / 3.0));
            const double tx = -ny, ty = nx, qt = 0.0;
            q_in_ex[0] = qi[0];
            q_in_ex[1] = qn * nx + qt * tx;
            q_in_ex[2] = qn * ny + qt * ty;
            q_ex_ex[0] = qe[0];
            q_ex_ex[1] = q_in_ex[1];
            q_ex_ex[2] = q_in_ex[2];
            if (!wet_ex) g_ex = 0.0;
        } else if (hi < he) {  // overtopping from ex to in
            const double mx = -nx, my = -ny;
            double qn;
            if (hi > 2.0 * he / 3.0)
                qn = Cs * hi * sqrt(2.0 * A.g * (he - hi));
            else
                qn = Cp * (2.0 * he / 3.0) * sqrt(A.g * (2.0 * he / 3.0));
            const double tx = -my, ty = mx, qt = 0.0;
            q_ex_ex[0] = qe[0];
            q_ex_ex[1] = qn * mx + qt * tx;
            q_ex_ex[2] = qn * my + qt * ty;
            q_in_ex[0] = qi[0];
            q_in_ex[1] = q_ex_ex[1];
            q_in_ex[2] = q_ex_ex[2];
            if (!wet_in) g_in = 0.0;
        }
        double Fi[3], Fe[3];
        llf_flux<double>(g_in, qi, q_in_ex, ti[3][g], D[2 + 9 + g], nx, ny, Fi);
        llf_flux<double>(g_ex, qe, q_ex_ex, te[3][ge], D[2 + 12 + ge], -nx, -ny, Fe);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            F[v * NG + g] = Fi[v];
            F[(3 + v) * NG + g] = Fe[v];
        }
    }
}

template <typename Real>
cudaError_t launch_levee(const LeveeArgs<Real>& A, int p, cudaStream_t s) {
    if (A.n <= 0) return cudaSuccess;
    const unsigned nb = (unsigned)((A.n + 127) / 128);
    if (p == 1)
        levee_kernel<1, Real><<<nb, 128, 0, s>>>(A);
    else
        levee_kernel<2, Real><<<nb, 128, 0, s>>>(A);
    return cudaGetLastError();
}

template cudaError_t launch_levee<float>(const LeveeArgs<float>&, int, cudaStream_t);
template cudaError_t launch_levee<double>(const LeveeArgs<double>&, int, cudaStream_t);

}  // namespace dgsw
