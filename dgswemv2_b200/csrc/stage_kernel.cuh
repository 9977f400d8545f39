// Fused RKDG stage kernel for sm_100a.
//
// One CTA owns one tile of TILE consecutive elements (device order = Morton order of centroids).
// Per stage it does, in three phases separated by __syncthreads:
//   1. element phase (thread = element): load the element's modes into registers and shared memory,
//      rebuild its geometry from the FP64 node coordinates, and accumulate the volume and source
//      integrals (Problem::volume_kernel + source_kernel, rkdg_swe_proc_volume.hpp:9-35,
//      rkdg_swe_proc_source.hpp:9-18);
//   2. edge phase (thread = edge of the tile's list): evaluate the numerical flux at the edge Gauss
//      points once per edge (interfaces: LLF + the wet/dry fix-ups of ISP::Internal,
//      rkdg_swe_is_internal.hpp:26-95; boundaries: BC::Land / BC::Function, rkdg_swe_bc_land.hpp:41-66,
//      rkdg_swe_bc_function.hpp:27-60) into shared memory. An edge between two tiles is evaluated by
//      both CTAs with the same code on the same inputs, so both see the same bits and F_ex = -F_in
//      holds exactly as in the reference;
//   3. element phase: subtract the edge contributions in the reference's interface/boundary order,
//      apply M^-1 and the SSP-RK stage combination (element.hpp:502-505,
//      explicit_ssp_rk_stepper.hpp:67-80), the wetting/drying kernel (swe_post_wet_dry.hpp:6-145,
//      its depth tests in FP64 in every precision) and the NaN scrutiny; write the next stage state.
// Modal state layout in HBM: component-major SoA, q[(var*ND + dof) * ne_pad + element].
#ifndef DGSW_STAGE_KERNEL_CUH
#define DGSW_STAGE_KERNEL_CUH

#include <cstdint>

#include "function_sets.h"
#include "rk_tables.h"

namespace dgsw {

template <typename Real>
struct DevTables {  // master tables of one polynomial order, in the kernel's precision
    Real phi[6 * 6];      // [dof][gp]
    Real dphi[2][6 * 6];  // [z][dof][gp]
    Real mz[2][6 * 6];    // [z][gp][dof]
    Real phiw[6 * 6];     // [gp][dof]
    double psi[3][6];     // [node][gp] (FP64: global coordinates of the volume points)
    Real fphi[3][6 * 3];  // [face][dof][gp]
    double fpsi[3][3][3]; // [face][node][gp]
    Real gw[3];
    double minv[6];
};


struct DevStatus {
    unsigned int nan_flag;
    unsigned int nan_ref_elem;  // smallest reference element index with a NaN
    unsigned int pad[2];
};

struct DevClock {
    double t;      // time at the start of the current step (ESSPRKStepper::t)
    long long step;
};

// Kernel arguments. The master tables travel by value inside the argument block, which the
// hardware serves from its constant bank: every table index in the kernel is a compile-time
// constant (face tables, indexed per thread, are copied to shared memory first).
template <typename Real>
struct StageArgs {
    DevTables<Real> T;
    const Real* qk[DGSW_RK_MAX_STAGES];  // stage states q_0..q_s used by this stage's combination
    const Real* solk[DGSW_RK_MAX_STAGES];
    double a[DGSW_RK_MAX_STAGES];
    double bdt[DGSW_RK_MAX_STAGES];
    int nterms;
    int store_sol;  // write sol_s (needed when a later stage uses it)
    Real* q_out;
    Real* sol_out;
    const Real* bath;        // [ND][ne_pad]
    const int* enodes;       // [3][ne_pad]
    const int2* eslot;       // [ne]
    const int4* edges;       // tile edge lists
    const int* tile_edge_off;
    const double2* xy;       // node coordinates
    const double* nz;        // node bathymetry depth (wet/dry vertex depths)
    const unsigned char* wet_in;
    unsigned char* wet_out;
    const int* ref_of_dev;
    double* baryctr;  // [3][ne_pad] barycentre values of the new state for the slope limiter, or null
    DevStatus* status;
    const DevClock* clock;
    double drk_s;  // stage-time offset of this stage (t + dt*drk[s])
    int ne;
    int ne_pad;
    double g;
    double h_o, h_o_thr;
    int fn_set;
    double fn_params[16];
    int spherical;
    double sp_cos_lat0, sp_R;
};

// ------------------------------------------------------------------------------------------------
// LLF flux, rkdg_swe_LLF_flux.hpp:7-60 (sp applied to the in-side normal flux only, as there)
// ------------------------------------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ void llf_flux(Real gravity, const Real qin[3], const Real qex[3], Real bath, Real sp,
                                         Real nx, Real ny, Real F[3]) {
    const Real h_in = qin[0] + bath;
    const Real ih_in = Real(1) / h_in;
    const Real u_in = qin[1] * ih_in;
    const Real v_in = qin[2] * ih_in;
    const Real h_ex = qex[0] + bath;
    const Real ih_ex = Real(1) / h_ex;
    const Real u_ex = qex[1] * ih_ex;
    const Real v_ex = qex[2] * ih_ex;
    const Real un_in = u_in * nx + v_in * ny;
    const Real un_ex = u_ex * nx + v_ex * ny;
    const Real spc = (nx * sp) * (nx * sp) + ny * ny;
    const Real lam = fmax(fabs(un_in) + sqrt(gravity * h_in * spc), fabs(un_ex) + sqrt(gravity * h_ex * spc));
    const Real pe_in = gravity * (qin[0] * qin[0] * Real(0.5) + qin[0] * bath);
    const Real pe_ex = gravity * (qex[0] * qex[0] * Real(0.5) + qex[0] * bath);
    const Real uuh_in = u_in * qin[1], vvh_in = v_in * qin[2], uvh_in = u_in * qin[2];
    const Real uuh_ex = u_ex * qex[1], vvh_ex = v_ex * qex[2], uvh_ex = u_ex * qex[2];
    const Real f0 = sp * qin[1] * nx + qin[2] * ny;
    const Real f1 = sp * (uuh_in + pe_in) * nx + uvh_in * ny;
    const Real f2 = sp * uvh_in * nx + (vvh_in + pe_in) * ny;
    const Real e0 = qex[1] * nx + qex[2] * ny;
    const Real e1 = (uuh_ex + pe_ex) * nx + uvh_ex * ny;
    const Real e2 = uvh_ex * nx + (vvh_ex + pe_ex) * ny;
    F[0] = Real(0.5) * (f0 + e0 + lam * (qin[0] - qex[0]));
    F[1] = Real(0.5) * (f1 + e1 + lam * (qin[1] - qex[1]));
    F[2] = Real(0.5) * (f2 + e2 + lam * (qin[2] - qex[2]));
}

// land boundary ghost state (normal momentum mirrored) + LLF, rkdg_swe_bc_land.hpp:68-86
template <typename Real>
__device__ __forceinline__ void land_flux(Real g, Real nx, Real ny, const Real qin[3], Real bath, Real sp, Real F[3]) {
    const Real tx = -ny, ty = nx;
    const Real qn_ex = -(qin[1] * nx + qin[2] * ny);
    const Real qt_ex = qin[1] * tx + qin[2] * ty;
    Real qex[3];
    qex[0] = qin[0];
    qex[1] = qn_ex * nx + qt_ex * tx;
    qex[2] = qn_ex * ny + qt_ex * ty;
    llf_flux<Real>(g, qin, qex, bath, sp, nx, ny, F);
}

// Wet/dry fix-ups of ISP::Internal (rkdg_swe_is_internal.hpp:47-90) for an interface whose LLF
// ze-flux exceeds 1e-12 in magnitude with one side dry. Out of line: taken on few edges only.
template <typename Real>
__device__ __noinline__ void wd_fixup(Real g, const Real* qi, const Real* qe, Real bi, Real be, Real sp, Real nx, Real ny,
                                      bool wa, bool wb, Real* Fi, Real* Fe) {
    if (Fi[0] > Real(1e-12)) {
        if (!wa) {  // water flowing from the dry in-side: zero flux there, reflective wall on the ex side
            Fi[0] = Fi[1] = Fi[2] = Real(0);
            land_flux<Real>(g, -nx, -ny, qe, be, sp, Fe);
        } else if (!wb) {  // water flowing into the dry ex-side: gravity-free LLF there
            llf_flux<Real>(Real(0), qe, qi, be, sp, -nx, -ny, Fe);
            Fe[0] = -Fi[0];
        }
    } else if (Fi[0] < Real(-1e-12)) {
        if (!wb) {
            Fe[0] = Fe[1] = Fe[2] = Real(0);
            land_flux<Real>(g, nx, ny, qi, bi, sp, Fi);
        } else if (!wa) {
            llf_flux<Real>(Real(0), qi, qe, bi, sp, nx, ny, Fi);
            Fi[0] = -Fe[0];
        }
    }
}

// analytic function sets evaluated out of line (one copy per kernel)
template <typename Real>
__device__ __noinline__ void fn_eval_dev(int id, const double* P, const dgsw_fn_time* T, int source, Real x, Real y,
                                         Real* out) {
    dgsw_fn_eval<Real>(id, P, *T, source, x, y, out);
}

// ------------------------------------------------------------------------------------------------
// wetting/drying of one p>=1 element on its vertex values, swe_post_wet_dry.hpp:6-145, in FP64.
// qv: modal state (first three modes carry the linear part); returns the new wet flag and writes
// the new modes back (higher modes are zeroed whenever the vertex values are re-projected, like
// ProjectLinearToBasis).
// ------------------------------------------------------------------------------------------------
template <int ND, typename Real>
__device__ __forceinline__ bool wetting_drying(Real (&qv)[3][ND], const double bv[3], double bath_min, double h_o,
                                               double thr, bool wet) {
    double z[3], qx[3], qy[3], h[3];
    // ProjectBasisToLinear through T_basis_linear (basis_dubiner_2D.cpp:213-234)
    {
        const double a = qv[0][0], b = qv[0][1], c = qv[0][2];
        z[0] = a - b - c;
        z[1] = a - b + c;
        z[2] = a + 2.0 * b;
        const double ax = qv[1][0], bx = qv[1][1], cx = qv[1][2];
        qx[0] = ax - bx - cx;
        qx[1] = ax - bx + cx;
        qx[2] = ax + 2.0 * bx;
        const double ay = qv[2][0], by = qv[2][1], cy = qv[2][2];
        qy[0] = ay - by - cy;
        qy[1] = ay - by + cy;
        qy[2] = ay + 2.0 * by;
    }
    int ndry = 0;
    for (int v = 0; v < 3; ++v) {
        h[v] = z[v] + bv[v];
        if (h[v] <= h_o + thr) ++ndry;
    }
    double h_avg = (0.0 + h[0] + h[1] + h[2]) / 3;
    if (h_avg <= thr) h_avg = thr;
    bool reproject = false, check = false;
    if (ndry == 0) {
        if (wet) return true;
        check = true;
    } else if (ndry == 3) {
        for (int v = 0; v < 3; ++v) {
            z[v] = h_avg - bv[v];
            qx[v] = 0.0;
            qy[v] = 0.0;
        }
        wet = false;
        reproject = true;
    } else {
        if (h_avg <= h_o + thr) {
            for (int v = 0; v < 3; ++v) {
                z[v] = h_avg - bv[v];
                qx[v] = 0.0;
                qy[v] = 0.0;
            }
        } else {
            // first minimum / first maximum, like std::min_element / std::max_element
            int hmin = 0, hmax = 0;
            for (int v = 1; v < 3; ++v) {
                if (h[v] < h[hmin]) hmin = v;
                if (h[v] > h[hmax]) hmax = v;
            }
            const int hmid = 3 - hmax - hmin;
            double ht[3];
            ht[hmin] = h_o;
            ht[hmid] = fmax(h_o, h[hmid] - (ht[hmin] - h[hmin]) / 2);
            ht[hmax] = h[hmax] - (ht[hmin] - h[hmin]) - (ht[hmid] - h[hmid]);
            for (int v = 0; v < 3; ++v) h[v] = ht[v];
            double dqx = 0, dqy = 0;
            int ndv = 0;
            for (int v = 0; v < 3; ++v)
                if (h[v] <= h_o + thr) {
                    ndv++;
                    dqx += qx[v];
                    dqy += qy[v];
                    qx[v] = 0.0;
                    qy[v] = 0.0;
                }
            for (int v = 0; v < 3; ++v) {
                z[v] = h[v] - bv[v];
                if (h[v] > h_o + thr) {
                    qx[v] += dqx / (3 - ndv);
                    qy[v] += dqy / (3 - ndv);
                }
            }
        }
        reproject = true;
        check = true;
    }
    if (check) {
        int hmax = 0;
        for (int v = 1; v < 3; ++v)
            if (h[v] > h[hmax]) hmax = v;
        if (z[hmax] > h_o - bath_min) {
            wet = true;
        } else {
            wet = false;
            for (int v = 0; v < 3; ++v) {
                qx[v] = 0.0;
                qy[v] = 0.0;
            }
            reproject = true;
        }
    }
    if (reproject) {
        // ProjectLinearToBasis through T_linear_basis (:236-257)
        const double* src[3] = {z, qx, qy};
        for (int var = 0; var < 3; ++var) {
            const double* s = src[var];
            qv[var][0] = (Real)(s[0] * (1.0 / 3.0) + s[1] * (1.0 / 3.0) + s[2] * (1.0 / 3.0));
            qv[var][1] = (Real)(s[0] * (-1.0 / 6.0) + s[1] * (-1.0 / 6.0) + s[2] * (1.0 / 3.0));
            qv[var][2] = (Real)(s[0] * (-1.0 / 2.0) + s[1] * (1.0 / 2.0));
#pragma unroll
            for (int k = 3; k < ND; ++k) qv[var][k] = Real(0);
        }
    }
    return wet;
}

// ------------------------------------------------------------------------------------------------
// the stage kernel
// ------------------------------------------------------------------------------------------------
template <int P>
struct Dims {
    static constexpr int ND = (P + 1) * (P + 2) / 2;
    static constexpr int NQ = (P == 1) ? 3 : 6;  // Dunavant degree 2p
    static constexpr int NG = P + 1;             // Gauss-Legendre points for degree 2p+1
};

// shared-memory layout of the stage kernel
template <int P, typename Real, bool WD>
struct Smem {
    static constexpr int ND = Dims<P>::ND, NG = Dims<P>::NG;
    static constexpr int NFC = (WD ? 2 : 1) * 3 * NG;  // flux components stored per edge
    static __host__ __device__ size_t al(size_t b) { return (b + 15) & ~size_t(15); }
    // section offsets (16-byte aligned)
    static __host__ __device__ size_t off_bath(int tile) { return al(sizeof(Real) * (size_t)3 * ND * tile); }
    static __host__ __device__ size_t off_F(int tile) { return off_bath(tile) + al(sizeof(Real) * (size_t)ND * tile); }
    static __host__ __device__ size_t off_sJ(int tile, int me) { return off_F(tile) + al(sizeof(Real) * (size_t)NFC * me); }
    static __host__ __device__ size_t off_tab(int tile, int me) { return off_sJ(tile, me) + al(sizeof(double) * (size_t)me); }
    static __host__ __device__ size_t off_node(int tile, int me) {
        return off_tab(tile, me) + al(sizeof(Real) * (size_t)(3 * ND * NG + NG));
    }
    static __host__ __device__ size_t off_wet(int tile, int me) { return off_node(tile, me) + al(sizeof(int) * (size_t)3 * tile); }
    static __host__ __device__ size_t off_flag(int tile, int me) { return off_wet(tile, me) + al((size_t)tile); }
    static __host__ __device__ size_t bytes(int tile, int me) { return off_flag(tile, me) + al((size_t)me); }
};

// resident CTAs per SM the register budget is sized for
template <int P, typename Real, int TILE>
struct MinBlocks {
    static constexpr int value = sizeof(Real) == 4 ? (TILE == 128 ? 4 : 2) : (TILE == 128 ? 3 : 1);
};

template <int P, typename Real, bool WD, bool FSRC, int TILE>
__global__ void __launch_bounds__(TILE, (MinBlocks<P, Real, TILE>::value)) rkdg_stage_kernel(const __grid_constant__ StageArgs<Real> A, int max_edges) {
    constexpr int ND = Dims<P>::ND, NQ = Dims<P>::NQ, NG = Dims<P>::NG;
    const DevTables<Real>& T = A.T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SM = Smem<P, Real, WD>;
    Real* sq = reinterpret_cast<Real*>(smem_raw);                                          // [3*ND][TILE]
    Real* sbath = reinterpret_cast<Real*>(smem_raw + SM::off_bath(TILE));                  // [ND][TILE]
    Real* sF = reinterpret_cast<Real*>(smem_raw + SM::off_F(TILE));                        // [NFC][max_edges]
    double* ssJ = reinterpret_cast<double*>(smem_raw + SM::off_sJ(TILE, max_edges));       // [max_edges]
    Real* sfphi = reinterpret_cast<Real*>(smem_raw + SM::off_tab(TILE, max_edges));       // [3][ND][NG]
    Real* sgw = sfphi + 3 * ND * NG;
    int* snode = reinterpret_cast<int*>(smem_raw + SM::off_node(TILE, max_edges));        // [3][TILE]
    unsigned char* swet = smem_raw + SM::off_wet(TILE, max_edges);
    unsigned char* sflag = smem_raw + SM::off_flag(TILE, max_edges);

    const int tile = blockIdx.x;
    const int e0 = tile * TILE;
    const int nloc = min(TILE, A.ne - e0);
    const int tid = threadIdx.x;
    const int d = e0 + tid;
    const bool active = tid < nloc;
    const double t_stage = A.clock->t + A.drk_s;  // ESSPRKStepper::GetTimeAtCurrentStage
    const Real g = (Real)A.g;
    const Real* __restrict__ qs = A.qk[A.nterms - 1];  // this stage's state
    const dgsw_fn_time FT = dgsw_fn_prepare(A.fn_set, A.fn_params, t_stage);

    // face tables are indexed by per-thread face numbers: keep them in shared memory
    for (int i = tid; i < 3 * ND * NG; i += TILE) sfphi[i] = T.fphi[i / (ND * NG)][i % (ND * NG)];
    if (tid < NG) sgw[tid] = T.gw[tid];

    Real rhs[3][ND];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < ND; ++k) rhs[v][k] = Real(0);
    double aJ = 1.0;
    bool wet = false;

    // ---------------- phase 1: element volume + source ----------------
    if (active) {
        const int n0 = A.enodes[d], n1 = A.enodes[A.ne_pad + d], n2 = A.enodes[2 * A.ne_pad + d];
        snode[tid] = n0;
        snode[TILE + tid] = n1;
        snode[2 * TILE + tid] = n2;
        const double2 p0 = A.xy[n0], p1 = A.xy[n1], p2 = A.xy[n2];
        // Jacobian of the straight triangle, shape_straighttriangle.cpp:95-137
        const double J00 = (p1.x - p0.x) / 2.0, J01 = (p2.x - p0.x) / 2.0;
        const double J10 = (p1.y - p0.y) / 2.0, J11 = (p2.y - p0.y) / 2.0;
        const double det = J00 * J11 - J10 * J01;
        aJ = fabs(det);
        const double invdet = 1.0 / det;
        const Real Ji00 = (Real)(J11 * invdet), Ji10 = (Real)(-J10 * invdet);
        const Real Ji01 = (Real)(-J01 * invdet), Ji11 = (Real)(J00 * invdet);
        Real q[3][ND], b[ND];
#pragma unroll
        for (int c = 0; c < 3 * ND; ++c) {
            const Real val = qs[c * A.ne_pad + d];
            q[c / ND][c % ND] = val;
            sq[c * TILE + tid] = val;
        }
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            b[k] = A.bath[k * A.ne_pad + d];
            sbath[k * TILE + tid] = b[k];
        }
        wet = A.wet_in[d] != 0;
        swet[tid] = wet ? 1 : 0;
        if (wet) {
            // unrolled: every table entry becomes an immediate constant-bank operand
#pragma unroll
            for (int gp = 0; gp < NQ; ++gp) {
                Real qg[3], bg = Real(0), db0 = Real(0), db1 = Real(0);
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    Real s = Real(0);
#pragma unroll
                    for (int k = 0; k < ND; ++k) s += q[v][k] * T.phi[k * NQ + gp];
                    qg[v] = s;
                }
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    bg += b[k] * T.phi[k * NQ + gp];
                    db0 += b[k] * T.dphi[0][k * NQ + gp];
                    db1 += b[k] * T.dphi[1][k * NQ + gp];
                }
                // physical flux, swe_flux.hpp:5-25
                const Real h = qg[0] + bg;
                const Real ih = Real(1) / h;
                const Real u = qg[1] * ih, vv = qg[2] * ih;
                const Real pe = g * (Real(0.5) * qg[0] * qg[0] + qg[0] * bg);
                Real Fx[3] = {qg[1], u * qg[1] + pe, u * qg[2]};
                Real Fy[3] = {qg[2], u * qg[2], vv * qg[2] + pe};
                double xg = 0.0, yg = 0.0;
                if (FSRC || A.spherical) {
                    xg = p0.x * T.psi[0][gp] + p1.x * T.psi[1][gp] + p2.x * T.psi[2][gp];
                    yg = p0.y * T.psi[0][gp] + p1.y * T.psi[1][gp] + p2.y * T.psi[2][gp];
                }
                if (A.spherical) {
                    const Real sp = (Real)(A.sp_cos_lat0 / cos(yg / A.sp_R));
#pragma unroll
                    for (int v = 0; v < 3; ++v) Fx[v] = sp * Fx[v];
                }
                // bathymetry-slope source, swe_source.hpp:15-21 (db/dx through J^-1)
                const Real dbx = db0 * Ji00 + db1 * Ji10;
                const Real dby = db0 * Ji01 + db1 * Ji11;
                Real S[3] = {Real(0), g * (dbx * qg[0]), g * (dby * qg[0])};
                if (FSRC) {
                    Real fs[3];
                    fn_eval_dev<Real>(A.fn_set, A.fn_params, &FT, 1, (Real)xg, (Real)yg, fs);
                    S[0] += fs[0];
                    S[1] += fs[1];
                    S[2] += fs[2];
                }
                // int F . grad(phi) = sum_gp sum_z (F_x J^-1(z,x) + F_y J^-1(z,y)) dphi_z w
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const Real G0 = Fx[v] * Ji00 + Fy[v] * Ji01;
                    const Real G1 = Fx[v] * Ji10 + Fy[v] * Ji11;
#pragma unroll
                    for (int k = 0; k < ND; ++k)
                        rhs[v][k] += G0 * T.mz[0][gp * ND + k] + G1 * T.mz[1][gp * ND + k] + S[v] * T.phiw[gp * ND + k];
                }
            }
            const Real raJ = (Real)aJ;
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) rhs[v][k] *= raJ;
        }
    }
    __syncthreads();

    // ---------------- phase 2: edge fluxes, once per edge of the tile ----------------
    const int eoff = A.tile_edge_off[tile];
    const int nedge = A.tile_edge_off[tile + 1] - eoff;
#pragma unroll 1
    for (int le = tid; le < nedge; le += TILE) {
        const int4 rec = A.edges[eoff + le];
        const int ea = rec.x, eb = rec.y;
        const int fa = rec.z & 3, fb = (rec.z >> 2) & 3, kind = (rec.z >> 4) & 3;
        const int la = ea - e0, lb = eb - e0;
        const bool a_loc = (la >= 0 && la < nloc), b_loc = (eb >= 0 && lb >= 0 && lb < nloc);
        const bool wa = a_loc ? swet[la] != 0 : A.wet_in[ea] != 0;
        const bool wb = (eb < 0) ? false : (b_loc ? swet[lb] != 0 : A.wet_in[eb] != 0);
        const bool compute = (kind == 0) ? (wa || wb) : wa;
        sflag[le] = compute ? 1 : 0;
        // face geometry from element a's vertices (fa+1)%3 -> (fa+2)%3
        const int va = (fa + 1) % 3, vb = (fa + 2) % 3;
        const int na = a_loc ? snode[va * TILE + la] : A.enodes[va * A.ne_pad + ea];
        const int nb = a_loc ? snode[vb * TILE + la] : A.enodes[vb * A.ne_pad + ea];
        const double2 pa = A.xy[na], pb = A.xy[nb];
        const double dx = pb.x - pa.x, dy = pb.y - pa.y;
        const double len = sqrt(dx * dx + dy * dy);
        ssJ[le] = len / 2.0;  // surface Jacobian = half edge length
        if (!compute) continue;
        const double ilen = 1.0 / len;
        const Real nx = (Real)(dy * ilen), ny = (Real)(-dx * ilen);  // outward unit normal of element a
        // traces at the edge Gauss points, accumulated over the modes in ascending order
        Real ti[3][NG], te[3][NG], bi[NG], be[NG];
#pragma unroll
        for (int gp = 0; gp < NG; ++gp) {
            ti[0][gp] = ti[1][gp] = ti[2][gp] = Real(0);
            te[0][gp] = te[1][gp] = te[2][gp] = Real(0);
            bi[gp] = be[gp] = Real(0);
        }
        const Real* fta = sfphi + fa * ND * NG;
        const Real* ftb = sfphi + fb * ND * NG;
#pragma unroll
        for (int k = 0; k < ND; ++k) {
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const Real c = a_loc ? sq[(v * ND + k) * TILE + la] : qs[(v * ND + k) * A.ne_pad + ea];
#pragma unroll
                for (int gp = 0; gp < NG; ++gp) ti[v][gp] += c * fta[k * NG + gp];
            }
            const Real c = a_loc ? sbath[k * TILE + la] : A.bath[k * A.ne_pad + ea];
#pragma unroll
            for (int gp = 0; gp < NG; ++gp) bi[gp] += c * fta[k * NG + gp];
        }
        if (kind == 0) {
#pragma unroll
            for (int k = 0; k < ND; ++k) {
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const Real c = b_loc ? sq[(v * ND + k) * TILE + lb] : qs[(v * ND + k) * A.ne_pad + eb];
#pragma unroll
                    for (int gp = 0; gp < NG; ++gp) te[v][gp] += c * ftb[k * NG + (NG - 1 - gp)];
                }
                if (WD) {
                    const Real c = b_loc ? sbath[k * TILE + lb] : A.bath[k * A.ne_pad + eb];
#pragma unroll
                    for (int gp = 0; gp < NG; ++gp) be[gp] += c * ftb[k * NG + (NG - 1 - gp)];
                }
            }
        }
        Real sp = Real(1);
        double xg[NG], yg[NG];
        if (kind == 2 || A.spherical) {
            const int m0 = a_loc ? snode[la] : A.enodes[ea];
            const int m1 = a_loc ? snode[TILE + la] : A.enodes[A.ne_pad + ea];
            const int m2 = a_loc ? snode[2 * TILE + la] : A.enodes[2 * A.ne_pad + ea];
            const double2 c0 = A.xy[m0], c1 = A.xy[m1], c2 = A.xy[m2];
#pragma unroll
            for (int gp = 0; gp < NG; ++gp) {
                xg[gp] = c0.x * T.fpsi[fa][0][gp] + c1.x * T.fpsi[fa][1][gp] + c2.x * T.fpsi[fa][2][gp];
                yg[gp] = c0.y * T.fpsi[fa][0][gp] + c1.y * T.fpsi[fa][1][gp] + c2.y * T.fpsi[fa][2][gp];
            }
        }
#pragma unroll
        for (int gp = 0; gp < NG; ++gp) {
            if (A.spherical) sp = (Real)(A.sp_cos_lat0 / cos(yg[gp] / A.sp_R));
            const Real qi[3] = {ti[0][gp], ti[1][gp], ti[2][gp]};
            Real qe[3];
            if (kind == 0) {
                qe[0] = te[0][gp];
                qe[1] = te[1][gp];
                qe[2] = te[2][gp];
            } else if (kind == 1) {
                // BC::Land ghost state: normal momentum mirrored (rkdg_swe_bc_land.hpp:44-56)
                const Real tx = -ny, ty = nx;
                const Real qn_ex = -(qi[1] * nx + qi[2] * ny);
                const Real qt_ex = qi[1] * tx + qi[2] * ty;
                qe[0] = qi[0];
                qe[1] = qn_ex * nx + qt_ex * tx;
                qe[2] = qn_ex * ny + qt_ex * ty;
            } else {
                // BC::Function ghost state: ic_q(t, x_gp) (rkdg_swe_bc_function.hpp:33-50)
                fn_eval_dev<Real>(A.fn_set, A.fn_params, &FT, 0, (Real)xg[gp], (Real)yg[gp], qe);
            }
            Real Fi[3];
            llf_flux<Real>(g, qi, qe, bi[gp], sp, nx, ny, Fi);
            if (WD && kind == 0) {
                Real Fe[3] = {-Fi[0], -Fi[1], -Fi[2]};
                if (!(wa && wb)) wd_fixup<Real>(g, qi, qe, bi[gp], be[gp], sp, nx, ny, wa, wb, Fi, Fe);
#pragma unroll
                for (int v = 0; v < 3; ++v) sF[((3 + v) * NG + gp) * max_edges + le] = Fe[v];
            }
#pragma unroll
            for (int v = 0; v < 3; ++v) sF[(v * NG + gp) * max_edges + le] = Fi[v];
        }
    }
    __syncthreads();

    // ---------------- phase 3: edge contributions, M^-1, RK combination, wet/dry ----------------
    if (!active) return;
    const int2 es = A.eslot[d];
    const int roles = es.y & 7;
    const int ord = es.y >> 3;
    const int cnt = ord & 3;
#pragma unroll 1
    for (int i = 0; i < cnt; ++i) {
        const int f = (ord >> (2 + 2 * i)) & 3;
        const int slot = (es.x >> (10 * f)) & 1023;
        if (!sflag[slot]) continue;
        const bool is_in = (roles >> f) & 1;
        const Real sJ = (Real)ssJ[slot];
        const Real* ft = sfphi + f * ND * NG;
#pragma unroll
        for (int gp = 0; gp < NG; ++gp) {  // own Gauss point order
            Real F[3];
            if (is_in) {
#pragma unroll
                for (int v = 0; v < 3; ++v) F[v] = sF[(v * NG + gp) * max_edges + slot];
            } else {
                const int ga = NG - 1 - gp;
#pragma unroll
                for (int v = 0; v < 3; ++v)
                    F[v] = WD ? sF[((3 + v) * NG + ga) * max_edges + slot] : -sF[(v * NG + ga) * max_edges + slot];
            }
            const Real wsJ = sgw[gp] * sJ;
#pragma unroll
            for (int k = 0; k < ND; ++k) {
                const Real ph = ft[k * NG + gp] * wsJ;
#pragma unroll
                for (int v = 0; v < 3; ++v) rhs[v][k] -= F[v] * ph;
            }
        }
    }
    // M^-1 (diagonal master mass inverse over |J|) and the SSP-RK stage combination
    const double iaJ = 1.0 / aJ;
    Real qn[3][ND];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            const Real sol = rhs[v][k] * (Real)(T.minv[k] * iaJ);
            const int idx = (v * ND + k) * A.ne_pad + d;
            if (A.store_sol) A.sol_out[idx] = sol;
            Real acc = Real(0);
            for (int j = 0; j < A.nterms - 1; ++j) {
                acc += (Real)A.a[j] * A.qk[j][idx];
                if (A.bdt[j] != 0.0) acc += (Real)A.bdt[j] * A.solk[j][idx];
            }
            const int j = A.nterms - 1;
            acc += (Real)A.a[j] * sq[(v * ND + k) * TILE + tid] + (Real)A.bdt[j] * sol;
            qn[v][k] = acc;
        }
    bool wet_new = wet;
    if (WD) {
        const double bv[3] = {A.nz[snode[tid]], A.nz[snode[TILE + tid]], A.nz[snode[2 * TILE + tid]]};
        const double bmin = fmin(bv[0], fmin(bv[1], bv[2]));
        wet_new = wetting_drying<ND, Real>(qn, bv, bmin, A.h_o, A.h_o_thr, wet);
    }
    bool has_nan = false;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            has_nan |= isnan((double)qn[v][k]);
            A.q_out[(v * ND + k) * A.ne_pad + d] = qn[v][k];
        }
    A.wet_out[d] = wet_new ? 1 : 0;
    if (A.baryctr) {
        // slope_limiting_prepare_element_kernel (swe_CS_slope_limiter.hpp:9-20): vertex values through
        // T_basis_linear, barycentre value = vertex values . (1/3, 1/3, 1/3)
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double a = qn[v][0], b = qn[v][1], c = qn[v][2];
            const double l0 = a - b - c, l1 = a - b + c, l2 = a + 2.0 * b;
            A.baryctr[v * A.ne_pad + d] = l0 * (1.0 / 3.0) + l1 * (1.0 / 3.0) + l2 * (1.0 / 3.0);
        }
    }
    if (has_nan) {
        atomicOr(&A.status->nan_flag, 1u);
        atomicMin(&A.status->nan_ref_elem, (unsigned int)A.ref_of_dev[d]);
    }
}

}  // namespace dgsw


namespace dgsw {
// launchers, one translation unit per (order, precision)
cudaError_t launch_stage_p1_f64(const StageArgs<double>& A, int tile, int ntiles, int max_edges, bool wd, bool fsrc,
                                cudaStream_t s);
cudaError_t launch_stage_p1_f32(const StageArgs<float>& A, int tile, int ntiles, int max_edges, bool wd, bool fsrc,
                                cudaStream_t s);
cudaError_t launch_stage_p2_f64(const StageArgs<double>& A, int tile, int ntiles, int max_edges, bool wd, bool fsrc,
                                cudaStream_t s);
cudaError_t launch_stage_p2_f32(const StageArgs<float>& A, int tile, int ntiles, int max_edges, bool wd, bool fsrc,
                                cudaStream_t s);

template <int P, typename Real, bool WD, bool FSRC, int TILE>
cudaError_t launch_stage_impl(const StageArgs<Real>& A, int ntiles, int max_edges, cudaStream_t s) {
    auto kern = rkdg_stage_kernel<P, Real, WD, FSRC, TILE>;
    const size_t smem = Smem<P, Real, WD>::bytes(TILE, max_edges);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)ntiles, TILE, smem, s>>>(A, max_edges);
    return cudaGetLastError();
}

template <int P, typename Real>
cudaError_t launch_stage_dispatch(const StageArgs<Real>& A, int tile, int ntiles, int max_edges, bool wd, bool fsrc,
                                  cudaStream_t s) {
#define DGSW_TILE_CASES(WD_, FS_)                                                    \
    switch (tile) {                                                                   \
        case 128:                                                                     \
            return launch_stage_impl<P, Real, WD_, FS_, 128>(A, ntiles, max_edges, s); \
        case 256:                                                                     \
            return launch_stage_impl<P, Real, WD_, FS_, 256>(A, ntiles, max_edges, s); \
        default:                                                                      \
            return cudaErrorInvalidValue;                                             \
    }
    if (wd) {
        if (fsrc) {
            DGSW_TILE_CASES(true, true)
        } else {
            DGSW_TILE_CASES(true, false)
        }
    } else {
        if (fsrc) {
            DGSW_TILE_CASES(false, true)
        } else {
            DGSW_TILE_CASES(false, false)
        }
    }
#undef DGSW_TILE_CASES
}
}  // namespace dgsw

#endif
