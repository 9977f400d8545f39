// KXRCF-type trouble indicator of the Cockburn-Shu limiter pass (check_trouble,
// source/problem/SWE/problem_slope_limiter/swe_trouble_check.hpp:6-116). The reference evaluates it in
// every limiter pass on the state the limiter is about to see but does not use the result; here it is
// computed only when a caller asks for it (dgsw_rkdg_set_trouble), for parity and diagnostics.
//
// Per element: over its interfaces with at least one wet side whose own-side integral of
// n . (row 0, row 1) of the trace is negative (the reference uses rows x = 0 and y = 1 of q_at_gp,
// i.e. ze and qx, and this keeps that), I += |int (h_own - h_neighbour)| and the face length joins the
// inflow perimeter; then, for wet elements with a non-empty inflow perimeter,
// I /= r^((p+1)/2) * perimeter * max vertex depth (r the circumradius) and the element is troubled if
// I > 1; the troubled set then grows by five neighbour layers (six marking passes in the reference).
#include <cuda_runtime.h>

#include "stage_kernel.cuh"
#include "trouble.cuh"

namespace dgsw {

// face f's outward unit normal, half length and length, as face_geometry (host_setup.cpp) builds them
__device__ __forceinline__ void face_normal(const double2 (&X)[3], int f, double& nx, double& ny, double& sJ,
                                            double& len) {
    const double2 a = X[(f + 1) % 3], b = X[(f + 2) % 3];
    const double dx = b.x - a.x, dy = b.y - a.y;
    const double J00 = (X[1].x - X[0].x) / 2.0, J01 = (X[2].x - X[0].x) / 2.0;
    const double J10 = (X[1].y - X[0].y) / 2.0, J11 = (X[2].y - X[0].y) / 2.0;
    const double det = J00 * J11 - J10 * J01;
    const double cw = det / fabs(det);
    len = hypot(dx, dy);
    nx = cw * dy / len;
    ny = -cw * dx / len;
    sJ = sqrt(dx * dx + dy * dy) / 2.0;
}

template <int P, int F, typename Real>
__device__ __forceinline__ void load_trace(const TroubleArgs<Real>& A, int e, double (&t)[4][MT<P>::NG]) {
    constexpr int ND = MT<P>::ND;
    const size_t Pp = (size_t)A.ne_pad;
    double q[3][ND], b[3];
#pragma unroll
    for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = A.q[c * Pp + e];
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] = (double)A.bath[k * Pp + e];
    face_trace<P, F, double>(q, b, t);
}

template <int P, typename Real>
__device__ __forceinline__ void load_trace_f(const TroubleArgs<Real>& A, int e, int f, double (&t)[4][MT<P>::NG]) {
    if (f == 0)
        load_trace<P, 0, Real>(A, e, t);
    else if (f == 1)
        load_trace<P, 1, Real>(A, e, t);
    else
        load_trace<P, 2, Real>(A, e, t);
}

__device__ __forceinline__ void element_nodes(const int* enodes, const double2* xy, size_t P, int e, double2 (&X)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) X[k] = xy[enodes[k * P + e]];
}

template <int P, typename Real>
__global__ void __launch_bounds__(128) trouble_kernel(const TroubleArgs<Real> A) {
    constexpr int NG = MT<P>::NG;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= A.ne) return;
    const size_t Pp = (size_t)A.ne_pad;
    const bool wet_e = A.wet[e] != 0;
    double2 X[3];
    element_nodes(A.enodes, A.xy, Pp, e, X);
    double I = 0.0, perim = 0.0;
    for (int f = 0; f < 3; ++f) {
        const int m = A.nbr[f * Pp + e];
        if (m < 0) continue;  // boundaries take no part
        if (!(wet_e || A.wet[m] != 0)) continue;
        const int fm = A.nbr_face[f * Pp + e];
        // the interface geometry of its "in" side (smaller element ID), negated for the other side
        double nx, ny, sJ, len;
        const bool is_in = A.ref_of_dev[e] < A.ref_of_dev[m];
        if (is_in) {
            face_normal(X, f, nx, ny, sJ, len);
        } else {
            double2 Y[3];
            element_nodes(A.enodes, A.xy, Pp, m, Y);
            face_normal(Y, fm, nx, ny, sJ, len);
            nx = -nx;
            ny = -ny;
        }
        double te[4][NG], tm[4][NG];
        load_trace_f<P, Real>(A, e, f, te);
        load_trace_f<P, Real>(A, m, fm, tm);
        double qn = 0.0;
#pragma unroll
        for (int g = 0; g < NG; ++g) qn += (nx * te[0][g] + ny * te[1][g]) * ((double)MT<P>::gw(g) * sJ);
        if (qn < 0.0) {
            double s = 0.0;
#pragma unroll
            for (int g = 0; g < NG; ++g) {
                const double he = te[0][g] + te[3][g], hm = tm[0][NG - 1 - g] + tm[3][NG - 1 - g];
                s += (he - hm) * ((double)MT<P>::gw(g) * sJ);
            }
            double own_len = len;
            if (!is_in) {
                double a, b, c;
                face_normal(X, f, a, b, c, own_len);
            }
            perim += own_len;
            I += fabs(s);
        }
    }
    unsigned char troubled = 0;
    if (wet_e && perim != 0.0) {
        double hmax = 0.0;
        const double z0 = A.q[0 * Pp + e], z1 = A.q[1 * Pp + e], z2 = A.q[2 * Pp + e];
        const double b0 = (double)A.bath[e], b1 = (double)A.bath[Pp + e], b2 = (double)A.bath[2 * Pp + e];
        const double zv[3] = {z0 - z1 - z2, z0 - z1 + z2, z0 + 2.0 * z1};
        const double bv[3] = {b0 - b1 - b2, b0 - b1 + b2, b0 + 2.0 * b1};
#pragma unroll
        for (int v = 0; v < 3; ++v) hmax = fmax(hmax, zv[v] + bv[v]);
        const double area = fabs((X[1].x - X[0].x) * (X[2].y - X[0].y) - (X[2].x - X[0].x) * (X[1].y - X[0].y)) / 2.0;
        double r = 1.0 / (4.0 * area);
#pragma unroll
        for (int s = 0; s < 3; ++s) r *= hypot(X[s].x - X[(s + 1) % 3].x, X[s].y - X[(s + 1) % 3].y);
        I /= (pow(r, (P + 1.0) / 2.0) * perim * hmax);
        troubled = I > 1.0 ? 1 : 0;
    }
    A.I[e] = I;
    A.flag[e] = troubled;
}

// one layer of growth: out = in or any neighbour in
__global__ void __launch_bounds__(256) trouble_grow_kernel(const unsigned char* __restrict__ in,
                                                           unsigned char* __restrict__ out, const int* __restrict__ nbr,
                                                           int ne, int ne_pad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    unsigned char v = in[e];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const int m = nbr[(size_t)f * ne_pad + e];
        if (m >= 0) v |= in[m];
    }
    out[e] = v;
}

template <typename Real>
cudaError_t launch_trouble(const TroubleArgs<Real>& A, int p, unsigned char* scratch, unsigned char* out,
                           cudaStream_t s) {
    if (A.ne <= 0) return cudaSuccess;
    const unsigned nb = (unsigned)((A.ne + 127) / 128);
    if (p == 1)
        trouble_kernel<1, Real><<<nb, 128, 0, s>>>(A);
    else
        trouble_kernel<2, Real><<<nb, 128, 0, s>>>(A);
    // five growth layers: flag -> scratch -> out -> scratch -> out -> ... ending in out
    const unsigned gb = (unsigned)((A.ne + 255) / 256);
    const unsigned char* src = A.flag;
    for (int k = 0; k < 5; ++k) {
        unsigned char* dst = (k % 2 == 0) ? out : scratch;
        trouble_grow_kernel<<<gb, 256, 0, s>>>(src, dst, A.nbr, A.ne, A.ne_pad);
        src = dst;
    }
    return cudaGetLastError();
}

template cudaError_t launch_trouble<float>(const TroubleArgs<float>&, int, unsigned char*, unsigned char*, cudaStream_t);
template cudaError_t launch_trouble<double>(const TroubleArgs<double>&, int, unsigned char*, unsigned char*,
                                            cudaStream_t);

}  // namespace dgsw
