// Cockburn-Shu TVB slope limiter in characteristic variables (CS_slope_limiter_serial,
// source/problem/SWE/problem_slope_limiter/swe_CS_sl_serial.hpp:9-23; kernels in
// swe_CS_slope_limiter.hpp:9-189; eigenvectors R, R^-1 in problem_jacobian/swe_jacobian.hpp:462-550;
// limiter geometry from problem_preprocessor/swe_pre_init_data.hpp:252-326).
//
// One thread per element, after the stage kernel has written the new state, the new wet flags and
// the barycentre values of every element. The FP64 path limits in FP64 (cs_limit_element); the FP32 path
// in FP32 arithmetic on FP64 differences (cs_limit_element_f32), arranged so that FP32 rounding cannot
// reach the write-back test, a relative change against 1e-12. The geometry (centroids, medians,
// alpha = A^-1 b, r^2) is precomputed once per handle from the FP64 node coordinates.
// The KXRCF trouble indicator the reference evaluates in the same pass (swe_trouble_check.hpp) does
// not feed the limiter there and is not evaluated here.
#ifndef DGSW_LIMITER_KERNEL_CUH
#define DGSW_LIMITER_KERNEL_CUH

#include <cuda_runtime.h>

namespace dgsw {

template <typename Real>
struct LimiterArgs {
    Real* q;                    // state to limit in place [(var*ND+dof)][ne_pad]
    const double* baryctr;      // [3][ne_pad]
    const unsigned char* wet;   // new wet flags
    const int* nbr;             // [3][ne_pad] neighbour (device index) or -2 - boundary type
    const int* enodes;          // [3][ne_pad]
    const double2* xy;
    const double* nz;
    unsigned char* limited;     // per element: 1 if its state was changed
    int ne, ne_pad;
    double g, M, nu;
    void* status;
    const int* ref_of_dev;
    // optional gating by the troubled-cell indicator
    const int* list;                 // visit only list[0 .. *list_count) (NULL: every element)
    const int* list_count;
    const unsigned char* gate;       // write back only where gate[e] != 0 (NULL: everywhere)
    unsigned long long* counters;    // [IND_LIMITED], [IND_MISSED] accumulators (NULL: none)
    const double* lgeo;              // precomputed limiter geometry [16][ne_pad] (NULL: computed here)
    const float* lgeo_f;             // its first 15 rows rounded to FP32, for the FP32 form (NULL: lgeo)
};

// Limiter geometry of element e (swe_pre_init_data.hpp:252-326): per median b (from the centroid to the
// midpoint of edge b) the coefficients alpha of the median in the basis of the centroid-to-neighbour-
// centroid vectors of faces b and b+1 (a boundary face mirrors the centroid across the edge), the unit
// median direction and its squared length; then the bathymetry at the barycentre.
// G = {al0, al1, nx, ny, r^2} x 3 medians, zb
constexpr int LIM_GEO = 16;

template <typename Real>
__device__ __forceinline__ void limiter_geometry(const LimiterArgs<Real>& L, int e, const int (&nb)[3],
                                                 double (&G)[LIM_GEO]) {
    const size_t P = (size_t)L.ne_pad;
    const int n0 = L.enodes[e], n1 = L.enodes[P + e], n2 = L.enodes[2 * P + e];
    const double2 X0 = L.xy[n0], X1 = L.xy[n1], X2 = L.xy[n2];
    const double X[3][2] = {{X0.x, X0.y}, {X1.x, X1.y}, {X2.x, X2.y}};
    const double cx = (X[0][0] + X[1][0] + X[2][0]) / 3.0, cy = (X[0][1] + X[1][1] + X[2][1]) / 3.0;
    double mid[3][2], nbc[3][2];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        mid[b][0] = (X[(b + 1) % 3][0] + X[(b + 2) % 3][0]) / 2.0;
        mid[b][1] = (X[(b + 1) % 3][1] + X[(b + 2) % 3][1]) / 2.0;
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        if (nb[f] >= 0) {
            const int m = nb[f];
            const double2 Y0 = L.xy[L.enodes[m]], Y1 = L.xy[L.enodes[P + m]], Y2 = L.xy[L.enodes[2 * P + m]];
            nbc[f][0] = (Y0.x + Y1.x + Y2.x) / 3.0;
            nbc[f][1] = (Y0.y + Y1.y + Y2.y) / 3.0;
        } else {
            nbc[f][0] = 2.0 * mid[f][0] - cx;
            nbc[f][1] = 2.0 * mid[f][1] - cy;
        }
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const int e1 = b, e2 = (b + 1) % 3;
        const double bx = mid[b][0] - cx, by = mid[b][1] - cy;
        const double nrm = sqrt(bx * bx + by * by);
        const double A00 = nbc[e1][0] - cx, A10 = nbc[e1][1] - cy, A01 = nbc[e2][0] - cx, A11 = nbc[e2][1] - cy;
        const double idet = 1.0 / (A00 * A11 - A10 * A01);
        G[5 * b] = (A11 * idet) * bx + (-A01 * idet) * by;
        G[5 * b + 1] = (-A10 * idet) * bx + (A00 * idet) * by;
        G[5 * b + 2] = bx / nrm;
        G[5 * b + 3] = by / nrm;
        G[5 * b + 4] = bx * bx + by * by;
    }
    G[15] = L.nz[n0] * (1.0 / 3.0) + L.nz[n1] * (1.0 / 3.0) + L.nz[n2] * (1.0 / 3.0);
}

// once per handle: the geometry of every element into lgeo [LIM_GEO][ne_pad], and, for the FP32 form, the
// medians' coefficients, directions and squared lengths rounded to FP32 into lgeo_f [LIM_GEO - 1][ne_pad]
// (the FP32 form does that arithmetic in FP32; the bathymetry at the barycentre stays FP64)
template <typename Real>
__global__ void __launch_bounds__(256) limiter_geometry_kernel(const LimiterArgs<Real> L, double* __restrict__ lgeo,
                                                               float* __restrict__ lgeo_f) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L.ne) return;
    const size_t P = (size_t)L.ne_pad;
    int nb[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) nb[f] = L.nbr[f * P + e];
    double G[LIM_GEO];
    limiter_geometry(L, e, nb, G);
#pragma unroll
    for (int i = 0; i < LIM_GEO; ++i) lgeo[i * P + e] = G[i];
    if (lgeo_f) {
#pragma unroll
        for (int i = 0; i < LIM_GEO - 1; ++i) lgeo_f[i * P + e] = (float)G[i];
    }
}

// the limiter decision for element e (1 if its state changes); the new state is written only if `write`
template <int ND, typename Real>
__device__ __forceinline__ unsigned char cs_limit_element(const LimiterArgs<Real>& L, int e, bool write) {
    const size_t P = (size_t)L.ne_pad;
    unsigned char lim = 0;
    // two rounds of loads: the own wet flag and the neighbours, then everything else at once (the
    // neighbours' wet flags and means, the own modes, mean and geometry), before the decision to look
    int nb[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) nb[f] = L.nbr[f * P + e];
    if (!L.wet[e]) return 0;
    bool ok = true;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        if (nb[f] >= 0) {
            ok = ok && (L.wet[nb[f]] != 0);
        } else {
            const int bt = -2 - nb[f];
            // land, tide, flow and function boundaries set wet_neigh to the element's own flag; faces
            // without a boundary object (outflow, an unpaired levee face) never set it and keep its
            // initial false
            ok = ok && (bt >= 0 && bt <= 3);  // DGSW_BC_LAND .. DGSW_BC_FUNCTION
        }
    }
    // own vertex values (T_basis_linear) and derived barycentre / midpoint values
    double ql[3][3], qb[3], qm[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const double a = (double)L.q[(v * ND + 0) * P + e], b = (double)L.q[(v * ND + 1) * P + e],
                     c = (double)L.q[(v * ND + 2) * P + e];
        ql[v][0] = a - b - c;
        ql[v][1] = a - b + c;
        ql[v][2] = a + 2.0 * b;
        qb[v] = L.baryctr[v * P + e];
        // chi_midpts (master_triangle.tpp:23-33): midpoint b is opposite vertex b
        qm[v][0] = ql[v][1] * 0.5 + ql[v][2] * 0.5;
        qm[v][1] = ql[v][0] * 0.5 + ql[v][2] * 0.5;
        qm[v][2] = ql[v][0] * 0.5 + ql[v][1] * 0.5;
    }
    // limiter geometry (precomputed once per handle by limiter_geometry_kernel, or built here)
    double G[LIM_GEO];
    if (L.lgeo) {
#pragma unroll
        for (int i = 0; i < LIM_GEO; ++i) G[i] = L.lgeo[i * P + e];
    } else {
        limiter_geometry(L, e, nb, G);
    }
    double qnb[3][3];
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int v = 0; v < 3; ++v) qnb[f][v] = nb[f] >= 0 ? L.baryctr[v * P + nb[f]] : qb[v];
    if (!ok) return 0;
    const double zb = G[15];
    const double h = qb[0] + zb;
    const double u = qb[1] / h, vv = qb[2] / h;
    const double c = sqrt(L.g * h);
    double delta[3][3];  // [var][bound]
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const int e1 = b, e2 = (b + 1) % 3;
        const double al0 = G[5 * b], al1 = G[5 * b + 1], nx = G[5 * b + 2], ny = G[5 * b + 3], rsq = G[5 * b + 4];
        const double un = u * nx + vv * ny;
        const double iR[3][3] = {{(c + un) / (2 * c), -nx / (2 * c), -ny / (2 * c)},
                                 {u * ny - vv * nx, -ny, nx},
                                 {(c - un) / (2 * c), nx / (2 * c), ny / (2 * c)}};
        const double R[3][3] = {{1.0, 0.0, 1.0}, {u - c * nx, -ny, u + c * nx}, {vv - c * ny, nx, vv + c * ny}};
        double dch[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double wm = 0, w0 = 0, w1 = 0, w2 = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                wm += iR[i][j] * qm[j][b];
                w0 += iR[i][j] * qb[j];
                w1 += iR[i][j] * qnb[e1][j];
                w2 += iR[i][j] * qnb[e2][j];
            }
            const double wt = wm - w0;
            const double wd = al0 * (w1 - w0) + al1 * (w2 - w0);
            if (fabs(wt) <= L.M * rsq)
                dch[i] = wt;
            else if (signbit(wt) == signbit(wd))
                dch[i] = copysign(1.0, wt) * fmin(fabs(wt), fabs(L.nu * wd));
            else
                dch[i] = 0.0;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) s += R[i][j] * dch[j];
            delta[i][b] = s;
        }
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const double dsum = delta[v][0] + delta[v][1] + delta[v][2];
        if (dsum != 0.0) {
            double pos = 0.0, neg = 0.0;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                pos += fmax(0.0, delta[v][b]);
                neg += fmax(0.0, -delta[v][b]);
            }
            const double tp = fmin(1.0, neg / pos), tn = fmin(1.0, pos / neg);
#pragma unroll
            for (int b = 0; b < 3; ++b) delta[v][b] = tp * fmax(0.0, delta[v][b]) - tn * fmax(0.0, -delta[v][b]);
        }
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        // vertex values = barycentre + delta * T, T = ones - 2 I (swe_data_slope_limit.hpp)
        double qv[3];
        qv[0] = qb[v] + (-delta[v][0] + delta[v][1] + delta[v][2]);
        qv[1] = qb[v] + (delta[v][0] - delta[v][1] + delta[v][2]);
        qv[2] = qb[v] + (delta[v][0] + delta[v][1] - delta[v][2]);
        double d2 = 0, n2 = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double dd = qv[k] - ql[v][k];
            d2 += dd * dd;
            n2 += ql[v][k] * ql[v][k];
        }
        if (sqrt(d2) / sqrt(n2) > 1.0e-12) {
            lim = 1;
            if (!write) continue;
            L.q[(v * ND + 0) * P + e] = (Real)(qv[0] * (1.0 / 3.0) + qv[1] * (1.0 / 3.0) + qv[2] * (1.0 / 3.0));
            L.q[(v * ND + 1) * P + e] = (Real)(qv[0] * (-1.0 / 6.0) + qv[1] * (-1.0 / 6.0) + qv[2] * (1.0 / 3.0));
            L.q[(v * ND + 2) * P + e] = (Real)(qv[0] * (-1.0 / 2.0) + qv[1] * (1.0 / 2.0));
#pragma unroll
            for (int k = 3; k < ND; ++k) L.q[(v * ND + k) * P + e] = Real(0);
        }
    }
    return lim;
}

// The same limiter with its characteristic arithmetic in FP32, for the FP32 path. Rounding noise must not
// reach the write-back test (relative change of the vertex values above 1e-12), so the pass works on
// deviations from the unlimited reconstruction: the differences it transforms (midpoint minus barycentre,
// neighbour minus own barycentre) are formed in FP64 before rounding to FP32; each characteristic slope's
// change dch - wt is exactly zero where the minmod keeps wt; the positivity rebalance acts on the sum of
// those changes (the unlimited deltas sum to zero); and the vertex change R (dch - wt) T, free of rounding
// where nothing was limited, is compared with 1e-12 of the vertex values. A changed element keeps its FP64
// mean (mode 0, which the rebalanced deltas leave unchanged) and gets its slope modes as FP64 plus the FP32
// correction; higher modes are zeroed as ProjectLinearToBasis does.
template <int ND, typename Real>
__device__ __forceinline__ unsigned char cs_limit_element_f32(const LimiterArgs<Real>& L, int e, bool write) {
    const size_t P = (size_t)L.ne_pad;
    // two rounds of loads, as in cs_limit_element
    int nb[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) nb[f] = L.nbr[f * P + e];
    if (!L.wet[e]) return 0;
    bool ok = true;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        if (nb[f] >= 0)
            ok = ok && (L.wet[nb[f]] != 0);
        else
            ok = ok && (-2 - nb[f] >= 0 && -2 - nb[f] <= 3);  // boundary objects: land .. function
    }
    float du[3][3], dn[3][3], nq[3];  // [bound][var] midpoint - barycentre, [face][var] neighbour - own, |ql|
    double qb[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const double a = (double)L.q[(v * ND + 0) * P + e], b = (double)L.q[(v * ND + 1) * P + e],
                     c = (double)L.q[(v * ND + 2) * P + e];
        const double l0 = a - b - c, l1 = a - b + c, l2 = a + 2.0 * b;
        qb[v] = L.baryctr[v * P + e];
        du[0][v] = (float)((l1 * 0.5 + l2 * 0.5) - qb[v]);
        du[1][v] = (float)((l0 * 0.5 + l2 * 0.5) - qb[v]);
        du[2][v] = (float)((l0 * 0.5 + l1 * 0.5) - qb[v]);
        nq[v] = (float)sqrt(l0 * l0 + l1 * l1 + l2 * l2);
    }
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int v = 0; v < 3; ++v) dn[f][v] = nb[f] >= 0 ? (float)(L.baryctr[v * P + nb[f]] - qb[v]) : 0.0f;
    float G[LIM_GEO - 1];
    double zb;
    if (L.lgeo_f) {
#pragma unroll
        for (int i = 0; i < LIM_GEO - 1; ++i) G[i] = L.lgeo_f[i * P + e];
        zb = L.lgeo[(LIM_GEO - 1) * P + e];
    } else {
        double Gd[LIM_GEO];
        if (L.lgeo) {
#pragma unroll
            for (int i = 0; i < LIM_GEO; ++i) Gd[i] = L.lgeo[i * P + e];
        } else {
            limiter_geometry(L, e, nb, Gd);
        }
#pragma unroll
        for (int i = 0; i < LIM_GEO - 1; ++i) G[i] = (float)Gd[i];
        zb = Gd[LIM_GEO - 1];
    }
    if (!ok) return 0;
    const float h = (float)(qb[0] + zb);
    const float ih = 1.0f / h;
    const float u = (float)qb[1] * ih, vv = (float)qb[2] * ih;
    const float c = sqrtf((float)L.g * h), i2c = 0.5f / c;
    const float M = (float)L.M, nu = (float)L.nu;
    float dd[3][3];  // [bound][var] change of the limited delta from the unlimited one
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const int e1 = b, e2 = (b + 1) % 3;
        const float al0 = G[5 * b], al1 = G[5 * b + 1], nx = G[5 * b + 2], ny = G[5 * b + 3], rsq = G[5 * b + 4];
        const float un = u * nx + vv * ny;
        const float iR[3][3] = {{(c + un) * i2c, -nx * i2c, -ny * i2c},
                                {u * ny - vv * nx, -ny, nx},
                                {(c - un) * i2c, nx * i2c, ny * i2c}};
        const float R[3][3] = {{1.0f, 0.0f, 1.0f}, {u - c * nx, -ny, u + c * nx}, {vv - c * ny, nx, vv + c * ny}};
        float ch[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float wt = 0.0f, w1 = 0.0f, w2 = 0.0f;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                wt += iR[i][j] * du[b][j];
                w1 += iR[i][j] * dn[e1][j];
                w2 += iR[i][j] * dn[e2][j];
            }
            const float wd = al0 * w1 + al1 * w2;
            float dch;
            if (fabsf(wt) <= M * rsq)
                dch = wt;
            else if (signbit(wt) == signbit(wd))
                dch = copysignf(1.0f, wt) * fminf(fabsf(wt), fabsf(nu * wd));
            else
                dch = 0.0f;
            ch[i] = dch - wt;
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) dd[b][v] = R[v][0] * ch[0] + R[v][1] * ch[1] + R[v][2] * ch[2];
    }
    unsigned char lim = 0;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        // positivity rebalance of the deltas du + dd (the unlimited deltas sum to zero)
        const float dsum = dd[0][v] + dd[1][v] + dd[2][v];
        if (dsum != 0.0f) {
            float d[3], pos = 0.0f, neg = 0.0f;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                d[b] = du[b][v] + dd[b][v];
                pos += fmaxf(0.0f, d[b]);
                neg += fmaxf(0.0f, -d[b]);
            }
            const float tp = fminf(1.0f, neg / pos), tn = fminf(1.0f, pos / neg);
#pragma unroll
            for (int b = 0; b < 3; ++b) dd[b][v] = (tp * fmaxf(0.0f, d[b]) - tn * fmaxf(0.0f, -d[b])) - du[b][v];
        }
        // change of the vertex values, (dd T)_k with T = ones - 2 I
        const float s = dd[0][v] + dd[1][v] + dd[2][v];
        const float x0 = s - 2.0f * dd[0][v], x1 = s - 2.0f * dd[1][v], x2 = s - 2.0f * dd[2][v];
        if (sqrtf(x0 * x0 + x1 * x1 + x2 * x2) > 1.0e-12f * nq[v]) {
            lim = 1;
            if (!write) continue;
            // the slope modes are read again here (L1 hits) rather than held in registers across the pass
            const double m1 = (double)L.q[(v * ND + 1) * P + e], m2 = (double)L.q[(v * ND + 2) * P + e];
            L.q[(v * ND + 1) * P + e] = (Real)(m1 + (double)((-x0 - x1 + 2.0f * x2) * (1.0f / 6.0f)));
            L.q[(v * ND + 2) * P + e] = (Real)(m2 + (double)((-x0 + x1) * 0.5f));
#pragma unroll
            for (int k = 3; k < ND; ++k) L.q[(v * ND + k) * P + e] = Real(0);
        }
    }
    return lim;
}

// One thread per visited element (every element, or the indicator's work list with a grid-stride loop).
// MB resident 256-thread blocks per SM: 2 (128 registers), 3 (80 registers and a few hundred bytes of
// spills) or 4 (64 registers, the FP32 form); measured on the bowl, 3 is 13 % faster than 2 at 524,288
// triangles and 2 is faster at 131,072
template <int ND, typename Real, int MB, bool F32 = false>
__global__ void __launch_bounds__(256, MB) cs_limiter_kernel(const LimiterArgs<Real> L) {
    const int n = L.list ? *L.list_count : L.ne;
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += stride) {  // block-uniform trip count
        const int i = i0 + threadIdx.x;
        bool applied = false, missed = false;
        if (i < n) {
            const int e = L.list ? L.list[i] : i;
            const bool write = !L.gate || L.gate[e];
            const bool lim = (F32 ? cs_limit_element_f32<ND, Real>(L, e, write) : cs_limit_element<ND, Real>(L, e, write)) != 0;
            applied = lim && write;
            missed = lim && !write;
            L.limited[e] = applied ? 1 : 0;
        }
        if (L.counters) {
            const unsigned ma = __ballot_sync(0xffffffffu, applied), mm = __ballot_sync(0xffffffffu, missed);
            if ((threadIdx.x & 31) == 0) {
                if (ma) atomicAdd(&L.counters[2], (unsigned long long)__popc(ma));
                if (mm) atomicAdd(&L.counters[3], (unsigned long long)__popc(mm));
            }
        }
    }
}

// grid: one block per 256 elements, or a persistent grid of `list_blocks` blocks over a work list;
// f32: the FP32-arithmetic form (the FP32 path). Large meshes run more blocks per SM with fewer registers:
// 3 (80 registers) for the FP64 form, 4 (64 registers) for the FP32 form, whose slope modes are re-read
// at write-back instead of held (measured on the 2.1 M-triangle bowl: FP32 step 0.520 -> 0.499 ms at 4
// against 3; FP64 0.757 -> 0.765 ms, so it stays at 3)
#ifndef DGSW_LIM_MB_BIG
#define DGSW_LIM_MB_BIG 3
#endif
#ifndef DGSW_LIM_MB_BIG_F32
#define DGSW_LIM_MB_BIG_F32 4
#endif
template <typename Real, bool F32>
void launch_limiter_kernel_t(const LimiterArgs<Real>& L, int p, cudaStream_t s, int blocks) {
    const bool big = L.ne >= (1 << 18);
    constexpr int MB = F32 ? DGSW_LIM_MB_BIG_F32 : DGSW_LIM_MB_BIG;
    if (p == 1) {
        if (big)
            cs_limiter_kernel<3, Real, MB, F32><<<blocks, 256, 0, s>>>(L);
        else
            cs_limiter_kernel<3, Real, 2, F32><<<blocks, 256, 0, s>>>(L);
    } else {
        if (big)
            cs_limiter_kernel<6, Real, MB, F32><<<blocks, 256, 0, s>>>(L);
        else
            cs_limiter_kernel<6, Real, 2, F32><<<blocks, 256, 0, s>>>(L);
    }
}

template <typename Real>
cudaError_t launch_limiter_kernel(const LimiterArgs<Real>& L, int p, cudaStream_t s, int list_blocks = 0,
                                  bool f32 = false) {
    const int blocks = L.list ? list_blocks : (L.ne + 255) / 256;
    if (blocks <= 0) return cudaSuccess;
    if (f32)
        launch_limiter_kernel_t<Real, true>(L, p, s, blocks);
    else
        launch_limiter_kernel_t<Real, false>(L, p, s, blocks);
    return cudaGetLastError();
}

}  // namespace dgsw

#endif
