// Fused RKDG stage kernel for sm_100a.
//
// One CTA owns one tile of TILE consecutive elements (device order = Morton order of centroids).
// Per RK stage it does, in three phases separated by __syncthreads:
//   1. element phase (thread = element): load the element's modes, accumulate the volume and source
//      integrals in registers (Problem::volume_kernel + source_kernel, rkdg_swe_proc_volume.hpp:9-35,
//      rkdg_swe_proc_source.hpp:9-18), and write the traces of its three faces at the edge Gauss points
//      to shared memory. Neighbours in other tiles ("halo" faces) get their face traces written by the
//      same routine from global memory;
//   2. edge phase (thread = edge of the tile's list): numerical flux at the edge Gauss points once per
//      edge from the shared-memory traces (interfaces: LLF + the wet/dry fix-ups of ISP::Internal,
//      rkdg_swe_is_internal.hpp:26-95; boundaries: BC::Land / BC::Function, rkdg_swe_bc_land.hpp:41-66,
//      rkdg_swe_bc_function.hpp:27-60). An edge between two tiles is evaluated by both CTAs with the
//      same code on the same bits, so F_ex = -F_in holds exactly as in the reference;
//   3. element phase: subtract the edge contributions in the reference's interface/boundary order,
//      apply M^-1 and the SSP-RK stage combination (element.hpp:502-505,
//      explicit_ssp_rk_stepper.hpp:67-80), the wetting/drying kernel (swe_post_wet_dry.hpp:6-145, its
//      depth tests in FP64 in every precision) and the NaN scrutiny; write the next stage state.
// The master tables are compile-time constants (tables_gen.h): every table entry is an immediate,
// zero entries are skipped and unit entries become additions.
// HBM layout: component-major SoA, q[(var*ND + dof) * ne_pad + element].
#ifndef DGSW_STAGE_KERNEL_CUH
#define DGSW_STAGE_KERNEL_CUH

#include <cstdint>

#include "../../include/dgsw_rkdg.h"
#include "function_sets.h"
#include "rk_tables.h"
#include "tables_gen.h"

namespace dgsw {

// compile-time loops
template <int N>
struct IC {
    static constexpr int value = N;
};
template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F&& f) {
    if constexpr (B < E) {
        f(IC<B>{});
        sfor<B + 1, E>(f);
    }
}

// packed FP32 arithmetic of sm_100 (one FFMA2 issue for two FMAs): a0 += x0 c0 and a1 += x1 c1. Each lane is
// an IEEE fma with the scalar fma's rounding. The kernels pair variables (ze with qx; qy with the bathymetry
// or alone) so that both lanes share one coefficient. Z0 / Z1 mark terms whose coefficient is a compile-time
// zero; they are left out, as the scalar loops leave them out.
template <bool Z0 = false, bool Z1 = false>
__device__ __forceinline__ void fma_pair(float& a0, float& a1, float x0, float x1, float c0, float c1) {
    if constexpr (!Z0 && !Z1) {
        const float2 r = __ffma2_rn(make_float2(x0, x1), make_float2(c0, c1), make_float2(a0, a1));
        a0 = r.x;
        a1 = r.y;
    } else if constexpr (!Z0) {
        a0 = __fmaf_rn(x0, c0, a0);
    } else if constexpr (!Z1) {
        a1 = __fmaf_rn(x1, c1, a1);
    }
}

// NaN scrutiny (scrutinize_solution after every stage, rkdg_swe_proc_serial_step.hpp:59-65): the reference
// stops at the first stage whose state holds a NaN and reports the first element (ascending ID) there.
// nan_key = (stage counter << 32) | reference element index, stage counter = step * stages + stage, kept
// as the minimum over all stages and elements of a batch: the first bad stage, then its smallest element.
struct DevStatus {
    unsigned long long nan_key;  // ~0 while no NaN has been seen
    unsigned int nan_flag;
    unsigned int pad;
};

struct DevClock {
    double t;  // time at the start of the current step (ESSPRKStepper::t)
    long long step;
};

// Real is the arithmetic type of the stage (FP32 bulk or FP64); the stage states and stored stage
// solutions are FP64 in both, so that the RK update does not accumulate FP32 rounding from stage to stage
template <typename Real>
struct StageArgs {
    const double* qk[DGSW_RK_MAX_STAGES];  // stage states used by this stage's combination, q_s last
    const double* solk[DGSW_RK_MAX_STAGES];
    double a[DGSW_RK_MAX_STAGES];
    double bdt[DGSW_RK_MAX_STAGES];
    int nterms;
    int store_sol;  // write sol_s (needed when a later stage uses it)
    double* q_out;
    double* sol_out;
    const Real* bath;           // [3][ne_pad] bathymetry modes of the linear part
    const Real* geo;            // [5][ne_pad] J^-1(0,0), J^-1(0,1), J^-1(1,0), J^-1(1,1), |J|
    const int* enodes;          // [3][ne_pad]
    const int2* eslot;          // [ne] edge slot per face, roles, accumulation order
    const int4* edges;          // tile edge lists: trace slot of a, trace slot of b (-1), meta, element a
    const Real* egeo;           // [3][n_edges]: outward unit normal of a (x, y), half length
    const int* tile_edge_off;
    const int2* halo;           // tile halo lists: (element, face)
    const int* tile_halo_off;
    const double2* xy;          // node coordinates
    const double* nz;           // node bathymetry depth (wet/dry vertex depths)
    const unsigned char* wet_in;
    unsigned char* wet_out;
    const int* ref_of_dev;
    double* baryctr;  // [3][ne_pad] barycentre values of the new state for the slope limiter, or null
    DevStatus* status;
    const DevClock* clock;
    double drk_s;  // stage-time offset of this stage (t + dt*drk[s])
    int stage_index, nstages;  // this stage and the stages per step (the NaN report's stage counter)
    int ne;
    int ne_pad;
    int n_edges;  // total edge records (stride of egeo)
    double g;
    double h_o, h_o_thr;
    int fn_set;
    double fn_params[16];
    int spherical;
    double sp_cos_lat0, sp_R;
    // bottom friction (swe_source.hpp:29-51): DGSW_FRICTION_NONE / CHEZY / MANNING
    int friction;
    double friction_cf;
    const Real* manning;  // [ne_pad] g n^2 per element (Manning)
    // tide / flow boundary forcing: per forced face its first constituent entry and count; per entry
    // frequency, forcing factor, equilibrium argument, amplitude[3] and phase[3] at the Gauss points
    const int2* fface;
    const double* fcon;
    int ramp_on;           // ramp_duration not almost zero
    double ramp_duration;  // days
    // levee interface fluxes of this stage, [n_levee][2][3][NG] (levee.cu): in side, then ex side
    const double* levF;
    unsigned char* went_dry;  // [ne] wet_dry_state.went_completely_dry of the last wet/dry pass, or null
    int reverse;              // visit the tiles in reverse order (grid = one CTA per tile)
    // Stage increments (the SPLIT kernels, FP32 arithmetic without wetting/drying, limiter or levees): the
    // carried state q_0 is kept compensated, as the unevaluated sum q0f + q0lo of two Real values (q0f the
    // rounding of q_0, q0lo the rounding of the remainder: a 48-bit significand), and each intermediate
    // stage state as its increment d_s = q_s - q_0 in Real. With sum_k a_sk = 1 the combination
    // q_{s+1} = sum_k a_sk q_k + dt b_sk L(q_k) becomes d_{s+1} = sum_k a_sk d_k + dt b_sk L(q_k) (d_0 = 0):
    // q_0 leaves it, so the increments round relative to their own small size. The last stage forms
    // q0f + q0lo + d_ns in FP64 and splits it again.
    const Real* dk[DGSW_RK_MAX_STAGES];     // increments of the combination's terms (null for q_0), d_s last
    const Real* dsolk[DGSW_RK_MAX_STAGES];  // stored stage solutions of the earlier terms, in Real
    const Real* q0f;                        // carried state, leading part: stage input q_s = q0f + d_s
    const Real* q0lo;                       // carried state, trailing part (read by the last stage)
    Real* d_out;                            // d_{s+1} (intermediate stages)
    Real* dsol_out;                         // this stage's solution, when a later stage reads it
    Real* q0f_out;                          // new carried state, leading part (last stage)
    Real* q0lo_out;                         // new carried state, trailing part (last stage)
    int last;                               // this is the step's last stage
};

constexpr int FORCE_STRIDE_DEV = 9;

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

// the same flux in packed FP32 (FFMA2 / FMUL2 / FADD2): the in side in lane x, the ex side in lane y, each
// lane the scalar formula above with its terms in the same order (sp on the in lane only)
__device__ __forceinline__ void llf_flux_packed(float gravity, const float qin[3], const float qex[3], float bath,
                                                float sp, float nx, float ny, float F[3]) {
    const float2 q0 = make_float2(qin[0], qex[0]), q1 = make_float2(qin[1], qex[1]), q2 = make_float2(qin[2], qex[2]);
    const float2 N = make_float2(nx, nx), M = make_float2(ny, ny), B = make_float2(bath, bath);
    const float2 h = __fadd2_rn(q0, B);
    const float2 ih = make_float2(1.0f / h.x, 1.0f / h.y);
    const float2 u = __fmul2_rn(q1, ih), v = __fmul2_rn(q2, ih);
    const float2 un = __ffma2_rn(v, M, __fmul2_rn(u, N));
    const float spc = (nx * sp) * (nx * sp) + ny * ny;
    const float2 gh = __fmul2_rn(make_float2(gravity, gravity), h);
    const float lam = fmaxf(fabsf(un.x) + sqrtf(gh.x * spc), fabsf(un.y) + sqrtf(gh.y * spc));
    const float2 pe = __fmul2_rn(make_float2(gravity, gravity),
                                 __ffma2_rn(q0, B, __fmul2_rn(__fmul2_rn(q0, q0), make_float2(0.5f, 0.5f))));
    const float2 uuh = __fmul2_rn(u, q1), vvh = __fmul2_rn(v, q2), uvh = __fmul2_rn(u, q2);
    const float2 spv = make_float2(sp, 1.0f);
    const float2 f0 = __ffma2_rn(q2, M, __fmul2_rn(__fmul2_rn(spv, q1), N));
    const float2 f1 = __ffma2_rn(uvh, M, __fmul2_rn(__fmul2_rn(spv, __fadd2_rn(uuh, pe)), N));
    const float2 f2 = __ffma2_rn(__fadd2_rn(vvh, pe), M, __fmul2_rn(__fmul2_rn(spv, uvh), N));
    F[0] = 0.5f * (f0.x + f0.y + lam * (qin[0] - qex[0]));
    F[1] = 0.5f * (f1.x + f1.y + lam * (qin[1] - qex[1]));
    F[2] = 0.5f * (f2.x + f2.y + lam * (qin[2] - qex[2]));
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

// both sides' fluxes of an interface Gauss point, returned by value from wd_fixup
template <typename Real>
struct Flux2 {
    Real i0, i1, i2, e0, e1, e2;
};

// Wet/dry fix-ups of ISP::Internal (rkdg_swe_is_internal.hpp:47-90) for an interface whose LLF
// ze-flux exceeds 1e-12 in magnitude with one side dry; the ex-side flux starts as -F. Out of line
// (taken on few edges only), with its arguments and results passed by value so that the call site
// keeps them in registers.
template <typename Real>
__device__ __noinline__ Flux2<Real> wd_fixup(Real g, Real qi0, Real qi1, Real qi2, Real qe0, Real qe1, Real qe2,
                                             Real bi, Real be, Real sp, Real nx, Real ny, bool wa, bool wb, Real F0,
                                             Real F1, Real F2) {
    const Real qi[3] = {qi0, qi1, qi2}, qe[3] = {qe0, qe1, qe2};
    Real Fi[3] = {F0, F1, F2}, Fe[3] = {-F0, -F1, -F2};
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
    return Flux2<Real>{Fi[0], Fi[1], Fi[2], Fe[0], Fe[1], Fe[2]};
}

// three values returned by value from the out-of-line helpers below: an output array passed by
// address would live in local memory at every call site
template <typename Real>
struct Val3 {
    Real v0, v1, v2;
};

// analytic function sets evaluated out of line (one copy per kernel); T points to the CTA's shared copy
template <typename Real>
__device__ __noinline__ Val3<Real> fn_eval_dev(int id, const double* P, const dgsw_fn_time* T, int source, Real x,
                                               Real y) {
    Real out[3];
    dgsw_fn_eval<Real>(id, P, *T, source, x, y, out);
    return Val3<Real>{out[0], out[1], out[2]};
}

// Ghost states of the boundaries with data, out of line (one call site per Gauss point):
// BC::Function (kind 2): ic_q(t, x_gp) (rkdg_swe_bc_function.hpp:33-50);
// BC::Tide (kind 3) and BC::Flow (kind 4) (rkdg_swe_bc_tide.hpp:73-100, rkdg_swe_bc_flow.hpp:72-102), in
// FP64 in both precisions: the forced value is
// sum_con ramp * forcing_fact * amplitude_gp * cos(frequency * t + (equilib_arg - phase_gp) * PI / 180)
// with the reference's PI = 3.14159265359 and ramp = tanh(2 (t / 86400) / ramp_duration)
// (ESSPRKStepper::operator++, explicit_ssp_rk_stepper.hpp:49-65; 1 without a ramp). A tide sets the
// ghost surface elevation to it and keeps the interior momentum; a flow keeps the interior elevation
// and sets the ghost momentum to it times the outward normal. fi is the face's forcing record.
template <typename Real>
__device__ __noinline__ Val3<Real> boundary_ghost(const StageArgs<Real>* Ap, const dgsw_fn_time* T, int kind,
                                                  int fi, int gp, double t, Real x, Real y, Real qi0, Real qi1,
                                                  Real qi2, Real nx, Real ny) {
    const StageArgs<Real>& A = *Ap;
    if (kind == 2) {
        Real qe[3];
        dgsw_fn_eval<Real>(A.fn_set, A.fn_params, *T, 0, x, y, qe);
        return Val3<Real>{qe[0], qe[1], qe[2]};
    }
    constexpr double REF_PI = 3.14159265359;
    const double ramp = A.ramp_on ? tanh(2.0 * (t / 86400.0) / A.ramp_duration) : 1.0;
    const int2 fc = A.fface[fi];
    double acc = 0.0;
    for (int c = 0; c < fc.y; ++c) {
        const double* r = A.fcon + (size_t)(fc.x + c) * FORCE_STRIDE_DEV;
        acc += ramp * r[1] * r[3 + gp] * cos(r[0] * t + (r[2] - r[6 + gp]) * REF_PI / 180.0);
    }
    if (kind == 4) return Val3<Real>{qi0, (Real)acc * nx, (Real)acc * ny};
    return Val3<Real>{(Real)acc, qi1, qi2};
}

// the Manning friction factor g n^2 / h^(1/3), bounded below by the Chezy coefficient (swe_source.hpp:37-42);
// h^(-1/3) through the reciprocal cube root (the reference's pow(h, 1/3) differs from cbrt by the
// rounding of 1/3, a few ulps)
template <typename Real>
__device__ __forceinline__ Real manning_cf(Real gn2, Real h, Real cf0) {
    Real cf = gn2 * rcbrt(h);
    if (cf < cf0) cf = cf0;
    return cf;
}

// The manufactured sine set's source terms inline, with its constants hoisted out of the quadrature
// loops (the same formulas as dgsw_fn_eval, function_sets.h); every other set goes through fn_eval_dev.
template <typename Real>
struct SineSrc {
    // ze = c1 P, qx = -c2 Q, qy = c2 R, zex = c3 Q, zey = -c3 R, zet = -c4 P, qxx = qyy = c5 P,
    // qxy = qyx = c5 S, qxt = -c6 Q, qyt = c6 R with P = sx cy, Q = cx cy, R = sx sy, S = cx sy
    Real k, c1, c2, c3, c5, c6, c0, g, H;  // c0 = 2 c5 - c4 (the continuity source)
    Real kpi;                              // k / pi = 2 / L
};

template <typename Real>
__device__ __forceinline__ SineSrc<Real> sine_src_prepare(const double* P, const dgsw_fn_time& T) {
    const double k = 2.0 * M_PI / P[0], A = P[1], w = T.s[2], B = P[1] * T.s[2] / (2.0 * k);
    const double st = T.s[0], ct = T.s[1];
    SineSrc<Real> S;
    S.k = (Real)k;
    S.kpi = (Real)(2.0 / P[0]);
    S.c1 = (Real)(A * ct);
    S.c2 = (Real)(B * st);
    S.c3 = (Real)(A * k * ct);
    S.c5 = (Real)(B * k * st);
    S.c6 = (Real)(B * w * ct);
    S.c0 = (Real)(2.0 * B * k * st - A * w * st);
    S.g = (Real)P[4];
    S.H = (Real)P[2];
    return S;
}

// sin and cos of k x: FP64 through sincospi(2 x / L), whose argument reduction is an exact rounding to an
// integer (sincos reduces by pi in several parts; the two differ by the rounding of 2 pi / L, a few 1e-16
// relative); FP32 through the range-reduced hardware sine/cosine
template <typename Real>
__device__ __forceinline__ void sine_src_sincos(const SineSrc<Real>& S, Real x, Real& s, Real& c) {
    if constexpr (sizeof(Real) == 8)
        sincospi(S.kpi * x, &s, &c);
    else
        dgsw_sincos(S.k * x, &s, &c);
}

// sin and cos of an angle a0 + e from s0 = sin a0, c0 = cos a0 and a small increment e (|e| <= 0.05), by the
// angle-addition identities with the Taylor series of sin e and cos e through e^9 / e^8 (remainder below
// 1e-19). FP64 elements evaluate sin and cos at their centroid and turn them to the quadrature points
// this way.
__device__ __forceinline__ void rotate_small(double s0, double c0, double e, double& s, double& c) {
    const double z = e * e;
    const double ce = 1.0 + z * (-1.0 / 2 + z * (1.0 / 24 + z * (-1.0 / 720 + z * (1.0 / 40320))));
    const double se = e * (1.0 + z * (-1.0 / 6 + z * (1.0 / 120 + z * (-1.0 / 5040 + z * (1.0 / 362880)))));
    s = s0 * ce + c0 * se;
    c = c0 * ce - s0 * se;
}

// the set's source at a point from sin / cos of k x and k y
template <typename Real>
__device__ __forceinline__ void sine_src_terms(const SineSrc<Real>& S, Real sx, Real cx, Real sy, Real cy,
                                               Real (&out)[3]) {
    const Real Pp = sx * cy, Q = cx * cy, R = sx * sy, Sq = cx * sy;
    const Real qx = -S.c2 * Q, qy = S.c2 * R;
    const Real zex = S.c3 * Q, zey = -S.c3 * R;
    const Real qxx = S.c5 * Pp, qxy = S.c5 * Sq;  // qyy = qxx, qyx = qxy
    const Real h = S.c1 * Pp + S.H;
    const Real ih = Real(1) / h;
    const Real ih2 = ih * ih;
    out[0] = S.c0 * Pp;
    out[1] = -S.c6 * Q + (Real(2) * qx * qxx * ih - qx * qx * zex * ih2) +
             ((qxy * qy + qx * qxx) * ih - qx * qy * zey * ih2) + S.g * h * zex;
    out[2] = S.c6 * R + ((qxx * qy + qx * qxy) * ih - qx * qy * zex * ih2) + (Real(2) * qy * qxx * ih - qy * qy * zey * ih2) +
             S.g * h * zey;
}

template <typename Real>
__device__ __forceinline__ void sine_src_eval(const SineSrc<Real>& S, Real x, Real y, Real (&out)[3]) {
    Real sx, cx, sy, cy;
    sine_src_sincos<Real>(S, x, sx, cx);
    sine_src_sincos<Real>(S, y, sy, cy);
    sine_src_terms<Real>(S, sx, cx, sy, cy, out);
}

// the sine set's source at one point, out of line; its constants are rebuilt from the set's parameters
// (kernel parameter space) and the stage's time factors (shared memory), so no pointer to a local
// value is taken
template <typename Real>
__device__ __noinline__ Val3<Real> sine_src_far(const double* params, const dgsw_fn_time* T, Real x, Real y) {
    const SineSrc<Real> S = sine_src_prepare<Real>(params, *T);
    Real out[3];
    sine_src_eval<Real>(S, x, y, out);
    return Val3<Real>{out[0], out[1], out[2]};
}

// ------------------------------------------------------------------------------------------------
// wetting/drying of one p>=1 element on its vertex values, swe_post_wet_dry.hpp:6-145, in FP64.
// qv: modal state (first three modes carry the linear part); returns the new wet flag and writes
// the new modes back (higher modes are zeroed whenever the vertex values are re-projected, like
// ProjectLinearToBasis).
// ------------------------------------------------------------------------------------------------
template <int ND, typename Real>
__device__ __forceinline__ bool wetting_drying(Real (&qv)[3][ND], const double bv[3], double bath_min, double h_o,
                                               double thr, bool wet, bool& went_dry) {
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
    went_dry = h_avg <= thr;  // wet_dry_state.went_completely_dry
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
            // first minimum / first maximum, like std::min_element / std::max_element (the values
            // are tracked beside the indices: an array indexed at run time would live in local memory;
            // here some vertices are dry and some are not, so hmin != hmax)
            int hmin = 0, hmax = 0;
            double hminv = h[0], hmaxv = h[0];
#pragma unroll
            for (int v = 1; v < 3; ++v) {
                if (h[v] < hminv) hmin = v, hminv = h[v];
                if (h[v] > hmaxv) hmax = v, hmaxv = h[v];
            }
            const int hmid = 3 - hmax - hmin;
            const double hmidv = hmid == 0 ? h[0] : (hmid == 1 ? h[1] : h[2]);
            const double tmin = h_o;
            const double tmid = fmax(h_o, hmidv - (tmin - hminv) / 2);
            const double tmax = hmaxv - (tmin - hminv) - (tmid - hmidv);
#pragma unroll
            for (int v = 0; v < 3; ++v) h[v] = v == hmin ? tmin : (v == hmax ? tmax : tmid);
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
        // z at the first maximum of h
        double hmaxv = h[0], zmax = z[0];
#pragma unroll
        for (int v = 1; v < 3; ++v)
            if (h[v] > hmaxv) hmaxv = h[v], zmax = z[v];
        if (zmax > h_o - bath_min) {
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
        auto project = [&](const double (&s)[3], int var) {
            qv[var][0] = (Real)(s[0] * (1.0 / 3.0) + s[1] * (1.0 / 3.0) + s[2] * (1.0 / 3.0));
            qv[var][1] = (Real)(s[0] * (-1.0 / 6.0) + s[1] * (-1.0 / 6.0) + s[2] * (1.0 / 3.0));
            qv[var][2] = (Real)(s[0] * (-1.0 / 2.0) + s[1] * (1.0 / 2.0));
#pragma unroll
            for (int k = 3; k < ND; ++k) qv[var][k] = Real(0);
        };
        project(z, 0);
        project(qx, 1);
        project(qy, 2);
    }
    return wet;
}

// ------------------------------------------------------------------------------------------------
// compile-time table access
// ------------------------------------------------------------------------------------------------
template <int P>
using MT = ct::Master<P>;

// trace of an element's face F at the edge Gauss points: ze, qx, qy and bathymetry,
// sum over the modes in ascending order (same arithmetic for tile and halo elements)
template <int P, int F, typename Real, bool PK = false>
__device__ __forceinline__ void face_trace(const Real (&q)[3][MT<P>::ND], const Real (&b)[3],
                                           Real (&t)[4][MT<P>::NG]) {
    constexpr int ND = MT<P>::ND, NG = MT<P>::NG;
    if constexpr (PK) {
        // packed FP32: (ze, qx) and (qy, bathymetry) share each mode's coefficient
        sfor<0, NG>([&](auto G) {
            constexpr int g = decltype(G)::value;
            Real s0 = Real(0), s1 = Real(0), s2 = Real(0), sb = Real(0);
            sfor<0, ND>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr double c = MT<P>::fphi((F * ND + k) * NG + g);
                if constexpr (c != 0.0) {
                    fma_pair(s0, s1, q[0][k], q[1][k], (Real)c, (Real)c);
                    if constexpr (k < 3)
                        fma_pair(s2, sb, q[2][k], b[k], (Real)c, (Real)c);
                    else
                        s2 = __fmaf_rn(q[2][k], (Real)c, s2);
                }
            });
            t[0][g] = s0, t[1][g] = s1, t[2][g] = s2, t[3][g] = sb;
        });
        return;
    }
    sfor<0, NG>([&](auto G) {
        constexpr int g = decltype(G)::value;
        sfor<0, 3>([&](auto V) {
            constexpr int v = decltype(V)::value;
            Real s = Real(0);
            sfor<0, ND>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr double c = MT<P>::fphi((F * ND + k) * NG + g);
                if constexpr (c != 0.0) s += q[v][k] * (Real)c;
            });
            t[v][g] = s;
        });
        Real sb = Real(0);
        sfor<0, 3>([&](auto K) {
            constexpr int k = decltype(K)::value;
            constexpr double c = MT<P>::fphi((F * ND + k) * NG + g);
            if constexpr (c != 0.0) sb += b[k] * (Real)c;
        });
        t[3][g] = sb;
    });
}

// the same trace for a face known only at run time, with the face's basis values from a [mode][gp] table:
// the halo faces of a warp belong to different faces, and one compile-time copy per face would split the
// warp. Entries that are zero on this face but not on another add a zero product (the sum is unchanged), so
// the values equal face_trace's bit for bit.
template <int P, typename Real, bool PK = false>
__device__ __forceinline__ void face_trace_rt(const Real (&q)[3][MT<P>::ND], const Real (&b)[3], const Real* cf,
                                              Real (&t)[4][MT<P>::NG]) {
    constexpr int ND = MT<P>::ND, NG = MT<P>::NG;
    if constexpr (PK) {
        sfor<0, NG>([&](auto G) {
            constexpr int g = decltype(G)::value;
            Real s0 = Real(0), s1 = Real(0), s2 = Real(0), sb = Real(0);
            sfor<0, ND>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr bool used = MT<P>::fphi((0 * ND + k) * NG + g) != 0.0 ||
                                      MT<P>::fphi((1 * ND + k) * NG + g) != 0.0 ||
                                      MT<P>::fphi((2 * ND + k) * NG + g) != 0.0;
                if constexpr (used) {
                    const Real c = cf[k * NG + g];
                    fma_pair(s0, s1, q[0][k], q[1][k], c, c);
                    if constexpr (k < 3)
                        fma_pair(s2, sb, q[2][k], b[k], c, c);
                    else
                        s2 = __fmaf_rn(q[2][k], c, s2);
                }
            });
            t[0][g] = s0, t[1][g] = s1, t[2][g] = s2, t[3][g] = sb;
        });
        return;
    }
    sfor<0, NG>([&](auto G) {
        constexpr int g = decltype(G)::value;
        sfor<0, 3>([&](auto V) {
            constexpr int v = decltype(V)::value;
            Real s = Real(0);
            sfor<0, ND>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr bool used = MT<P>::fphi((0 * ND + k) * NG + g) != 0.0 ||
                                      MT<P>::fphi((1 * ND + k) * NG + g) != 0.0 ||
                                      MT<P>::fphi((2 * ND + k) * NG + g) != 0.0;
                if constexpr (used) s += q[v][k] * cf[k * NG + g];
            });
            t[v][g] = s;
        });
        Real sb = Real(0);
        sfor<0, 3>([&](auto K) {
            constexpr int k = decltype(K)::value;
            constexpr bool used = MT<P>::fphi((0 * ND + k) * NG + g) != 0.0 ||
                                  MT<P>::fphi((1 * ND + k) * NG + g) != 0.0 ||
                                  MT<P>::fphi((2 * ND + k) * NG + g) != 0.0;
            if constexpr (used) sb += b[k] * cf[k * NG + g];
        });
        t[3][g] = sb;
    });
}

// shared-memory layout of the stage kernel
template <int P, typename Real, bool WD>
struct Smem {
    static constexpr int ND = MT<P>::ND, NG = MT<P>::NG;
    static constexpr int NTC = 4 * NG;                 // trace components per face slot
    static constexpr int NFC = (WD ? 2 : 1) * 3 * NG;  // flux components stored per edge
    static __host__ __device__ size_t al(size_t b) { return (b + 15) & ~size_t(15); }
    static __host__ __device__ int nslot(int tile, int mh) { return 3 * tile + mh; }
    static __host__ __device__ size_t off_tr(int) { return 0; }
    static __host__ __device__ size_t off_F(int tile, int mh) {
        return off_tr(tile) + al(sizeof(Real) * (size_t)NTC * nslot(tile, mh));
    }
    static __host__ __device__ size_t off_sJ(int tile, int mh, int me) {
        return off_F(tile, mh) + al(sizeof(Real) * (size_t)NFC * me);
    }
    static __host__ __device__ size_t off_wet(int tile, int mh, int me) {
        return off_sJ(tile, mh, me) + al(sizeof(Real) * (size_t)me);
    }
    static __host__ __device__ size_t off_flag(int tile, int mh, int me) {
        return off_wet(tile, mh, me) + al((size_t)nslot(tile, mh));
    }
    // halo staging: the state and bathymetry modes of each halo face's element, copied asynchronously
    static __host__ __device__ size_t off_halo(int tile, int mh, int me) { return off_flag(tile, mh, me) + al((size_t)me); }
    static __host__ __device__ size_t off_hbath(int tile, int mh, int me) {
        return off_halo(tile, mh, me) + al(sizeof(double) * (size_t)3 * ND * mh);
    }
    static __host__ __device__ size_t bytes(int tile, int mh, int me) {
        return off_hbath(tile, mh, me) + al(sizeof(Real) * (size_t)3 * mh);
    }
};

// asynchronous global -> shared copies of one 4- or 8-byte value (the thread does not wait for it)
template <typename Real>
__device__ __forceinline__ void cp_async_value(Real* dst, const Real* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(Real) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_and_wait() {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// resident CTAs per SM the register budget is sized for (p = 1 and p = 2 separately; measured at tile
// 128 on 524,288 triangles: p = 2 FP32 4 (5 spills 592 B and runs 40 % slower), p = 1 FP32 5 (3-9 %
// faster than 4 on the bowl, tidal, levee and manufactured workloads; 6 spills and is slower), p = 2
// FP64 3, p = 1 FP64 4 without wetting/drying (14-15 % faster than 3 on the tidal, levee and
// manufactured workloads) and 3 with it (4 spills in the wet/dry pass and is 6 % slower on the bowl))
#ifndef DGSW_F32_MB128
#define DGSW_F32_MB128 4
#endif
#ifndef DGSW_F64_MB128
#define DGSW_F64_MB128 3
#endif
#ifndef DGSW_F32_P1_MB128
#define DGSW_F32_P1_MB128 5
#endif
#ifndef DGSW_F64_P1_MB128
#define DGSW_F64_P1_MB128 4
#endif
#ifndef DGSW_F64_P1_WD_MB128
#define DGSW_F64_P1_WD_MB128 3
#endif
// OCC = 1 selects the autotuner's alternative budget: one resident CTA fewer where the default holds
// several (more registers per thread), one more where it holds one (tile 256 in FP64)
template <int P, typename Real, int TILE, bool WD, int OCC = 0>
struct MinBlocks {
    static constexpr int f32 = P == 1 ? DGSW_F32_P1_MB128 : DGSW_F32_MB128;
    static constexpr int f64 = P == 1 ? (WD ? DGSW_F64_P1_WD_MB128 : DGSW_F64_P1_MB128) : DGSW_F64_MB128;
    static constexpr int base = sizeof(Real) == 4 ? (TILE == 128 ? f32 : 2) : (TILE == 128 ? f64 : 1);
    static constexpr int value = OCC == 0 ? base : (base > 1 ? base - 1 : base + 1);
};

// shared-memory capacities a tile almost always fits (measured: about 0.27 TILE halo faces and 1.65 TILE
// edges on structured and jittered meshes); with CAPPED the trace and flux strides are these
// compile-time constants, so every shared-memory access has an immediate offset
template <int TILE>
struct TileCap {
    static constexpr int halo = TILE / 2;
    static constexpr int edges = TILE + TILE / 2 + TILE / 4 + 16;  // 240 for 128, 464 for 256
};

template <int P, typename Real, bool WD, bool FSRC, bool FRIC, int TILE, bool CAPPED, int OCC = 0, bool SPLIT = false>
__global__ void __launch_bounds__(TILE, (MinBlocks<P, Real, TILE, WD, OCC>::value))
    rkdg_stage_kernel(const __grid_constant__ StageArgs<Real> A, int max_halo_rt, int max_edges_rt) {
    static_assert(!SPLIT || (!WD && sizeof(Real) == 4), "stage increments: FP32 arithmetic without wetting/drying");
    const int max_halo = CAPPED ? TileCap<TILE>::halo : max_halo_rt;
    const int max_edges = CAPPED ? TileCap<TILE>::edges : max_edges_rt;
    constexpr int ND = MT<P>::ND, NQ = MT<P>::NQ, NG = MT<P>::NG;
    using SM = Smem<P, Real, WD>;
    const int NS = SM::nslot(TILE, max_halo);  // trace slots: 3 per tile element, then halo faces
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // trace slots: FP32 at p = 2 [NS][NG][ze, qx, qy, b], one 16-byte shared access per Gauss point (a slot is
    // 36 words, so the 8 threads of a quarter-warp that write consecutive slots hit distinct banks);
    // otherwise [4*NG][NS]. Measured per step against [4*NG][NS] (same bits): config 2 -1.9 %, tidal p = 2
    // -1.4 %; at p = 1 (24-word slots, two-way bank conflicts) +1.3 to +1.5 %, so p = 1 keeps the old layout
    Real* str = reinterpret_cast<Real*>(smem_raw + SM::off_tr(TILE));
    constexpr bool tr_vec = sizeof(Real) == 4 && P == 2;
    auto tr_at = [&](int c, int gp, int slot) -> Real& {
        return tr_vec ? str[(slot * NG + gp) * 4 + c] : str[(c * NG + gp) * NS + slot];
    };
    // a face's traces into its slot
    auto put_trace = [&](int slot, const Real (&t)[4][NG]) {
        if constexpr (tr_vec) {
#pragma unroll
            for (int gg = 0; gg < NG; ++gg)
                *reinterpret_cast<float4*>(str + (slot * NG + gg) * 4) = make_float4(t[0][gg], t[1][gg], t[2][gg], t[3][gg]);
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int gg = 0; gg < NG; ++gg) str[(c * NG + gg) * NS + slot] = t[c][gg];
        }
    };
    Real* sF = reinterpret_cast<Real*>(smem_raw + SM::off_F(TILE, max_halo));       // [NFC][max_edges]
    Real* ssJ = reinterpret_cast<Real*>(smem_raw + SM::off_sJ(TILE, max_halo, max_edges));
    unsigned char* swet = smem_raw + SM::off_wet(TILE, max_halo, max_edges);        // [NS]
    unsigned char* sflag = smem_raw + SM::off_flag(TILE, max_halo, max_edges);      // [max_edges]
    double* shq = reinterpret_cast<double*>(smem_raw + SM::off_halo(TILE, max_halo, max_edges));  // [3*ND][max_halo]
    Real* shb = reinterpret_cast<Real*>(smem_raw + SM::off_hbath(TILE, max_halo, max_edges));      // [3][max_halo]

    // odd stages walk the tiles backwards: they start on the tiles the previous stage wrote last,
    // whose states are still in L2 (tiles are independent, so the results do not change)
    const int tile = A.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int e0 = tile * TILE;
    const int nloc = min(TILE, A.ne - e0);
    const int tid = threadIdx.x;
    const int d = e0 + tid;
    const bool active = tid < nloc;
    const int P_ = A.ne_pad;
    const double t_stage = A.clock->t + A.drk_s;  // ESSPRKStepper::GetTimeAtCurrentStage
    const Real g = (Real)A.g;
    const double* __restrict__ qs = A.qk[A.nterms - 1];  // this stage's state
    // the stage's time factors, once per CTA in shared memory (the out-of-line helpers read them there)
    __shared__ dgsw_fn_time sFT;
    if (threadIdx.x == 0) sFT = dgsw_fn_prepare(A.fn_set, A.fn_params, t_stage);
    // the face traces' basis values at the edge Gauss points, [face][mode][gp], for phase 3's lift and the
    // halo traces: the elements of a warp visit their faces in different orders, and compile-time tables per
    // face split the warp into one branch per face. Measured per step (bit-identical results): FP32 at p = 2
    // -0.6 to -0.9 %; FP64 at p = 2 -0.6 to +0.5 %, p = 1 +1 to +4 % (the shared-memory loads cost more than
    // the divergence there), so only FP32 at p = 2 uses it
    constexpr bool rt_face = P == 2 && sizeof(Real) == 4;
    // packed FP32 FMAs (fma_pair) in the Gauss-point state evaluation, the face traces, the volume integral and
    // the lift. Measured per step against the scalar FMAs: config 2 -4.5 %, the tidal channel -3.6 % (p = 2)
    // and -2 % (p = 1); warp instructions per config-2 stage -8 %. With wetting/drying (p = 1 bowl) the
    // scalar form stays: packed, the bowl step took 6 % longer.
    constexpr bool packed = sizeof(Real) == 4 && !WD;
    __shared__ Real sfphi[3 * ND * NG];
    if (rt_face && threadIdx.x < 3 * ND * NG) {
        Real c = Real(0);
        sfor<0, 3 * ND * NG>([&](auto I) {
            constexpr int i = decltype(I)::value;
            if (threadIdx.x == i) c = (Real)MT<P>::fphi(i);
        });
        sfphi[threadIdx.x] = c;
    }
    __syncthreads();
    const dgsw_fn_time& FT = sFT;
    // the manufactured sine set's source inline, in both precisions; other sets go through fn_eval_dev
    const bool sine_set = FSRC && A.fn_set == DGSW_FN_MANUFACTURED_SINE;
    SineSrc<Real> SS;
    if (sine_set) SS = sine_src_prepare<Real>(A.fn_params, FT);

    Real rhs[3][ND];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < ND; ++k) rhs[v][k] = Real(0);
    // stage increments: the combination's increment terms sum_k a_k d_k + dt b_k sol_k in Real, loaded at
    // the start of phase 3 (measured: issuing them before the first barrier instead gained nothing on the
    // p = 2 manufactured and tidal workloads and cost 3 % at p = 1)
    Real dcomb[3][ND];
    auto split_comb = [&]() {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < ND; ++k) dcomb[v][k] = Real(0);
        for (int j = 0; j < A.nterms; ++j) {
            const Real* __restrict__ dj = A.dk[j];
            if (dj) {
                const Real aj = (Real)A.a[j];
                Real t[3][ND];
#pragma unroll
                for (int v = 0; v < 3; ++v)
#pragma unroll
                    for (int k = 0; k < ND; ++k) t[v][k] = dj[(v * ND + k) * P_ + d];
                if constexpr (packed) {
#pragma unroll
                    for (int k = 0; k < ND; ++k) {
                        fma_pair(dcomb[0][k], dcomb[1][k], t[0][k], t[1][k], aj, aj);
                        dcomb[2][k] = __fmaf_rn(t[2][k], aj, dcomb[2][k]);
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < 3; ++v)
#pragma unroll
                        for (int k = 0; k < ND; ++k) dcomb[v][k] += aj * t[v][k];
                }
            }
            if (j < A.nterms - 1 && A.bdt[j] != 0.0) {
                const Real* __restrict__ sj = A.dsolk[j];
                const Real bj = (Real)A.bdt[j];
                Real u[3][ND];
#pragma unroll
                for (int v = 0; v < 3; ++v)
#pragma unroll
                    for (int k = 0; k < ND; ++k) u[v][k] = sj[(v * ND + k) * P_ + d];
                if constexpr (packed) {
#pragma unroll
                    for (int k = 0; k < ND; ++k) {
                        fma_pair(dcomb[0][k], dcomb[1][k], u[0][k], u[1][k], bj, bj);
                        dcomb[2][k] = __fmaf_rn(u[2][k], bj, dcomb[2][k]);
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < 3; ++v)
#pragma unroll
                        for (int k = 0; k < ND; ++k) dcomb[v][k] += bj * u[v][k];
                }
            }
        }
    };
    Real aJ = Real(1);
    bool wet = false;
    // this element's edge slots for phase 3, loaded now so that the latency is hidden
    const int2 es = active ? A.eslot[d] : make_int2(0, 0);
    // with capped tiles (at most TILE / 2 halo faces) thread h < nh owns halo face h: its record is
    // loaded now and its element's data copied asynchronously into shared memory during phase 1
    const int hoff = A.tile_halo_off[tile];
    const int nh = A.tile_halo_off[tile + 1] - hoff;
    const int eoff = A.tile_edge_off[tile];
    const int nedge = A.tile_edge_off[tile + 1] - eoff;
    // FP64: one thread asks L2 for the rows this CTA reads only after phase 1: the RK combination's
    // earlier stages (phase 3) and the tile's edge records and edge geometry (phase 2), so that those
    // phases start on L2 hits instead of HBM latency. Bulk prefetches want 16-byte aligned ranges: state
    // rows start on a multiple of TILE elements, the edge geometry rows are trimmed to whole 16-byte
    // blocks. Measured on 524,288 triangles: FP64 p = 2 stage 201 -> 199 us (tile 128) and 210 -> 206 us
    // (tile 256), the config-4 bowl 326 -> 309 us; the FP32 stages were unchanged or up to 2 % slower,
    // so they do without.
    if (sizeof(Real) == 8 && tid == 0) {
        auto prefetch = [](const void* p, unsigned bytes) {
            if (bytes >= 16)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes & ~15u) : "memory");
        };
        const unsigned rowb = (unsigned)((nloc + 1) & ~1) * 8u;
        for (int j = 0; j < A.nterms - 1; ++j) {
            for (int c = 0; c < 3 * ND; ++c) prefetch(A.qk[j] + (size_t)c * P_ + e0, rowb);
            if (A.bdt[j] != 0.0)
                for (int c = 0; c < 3 * ND; ++c) prefetch(A.solk[j] + (size_t)c * P_ + e0, rowb);
        }
        prefetch(A.edges + eoff, (unsigned)nedge * 16u);
        constexpr int per16 = 16 / (int)sizeof(Real);
        for (int c = 0; c < 3; ++c) {
            const int b = c * A.n_edges + eoff, e = b + nedge;
            const int b16 = (b + per16 - 1) / per16 * per16, e16 = e / per16 * per16;
            if (e16 > b16) prefetch(A.egeo + b16, (unsigned)(e16 - b16) * (unsigned)sizeof(Real));
        }
    }
    // stage increments, last stage: the carried state's trailing part is read only in the epilogue; one
    // thread asks L2 for this tile's rows now, so that those loads start on L2 hits
    if constexpr (SPLIT) {
        if (A.last && tid == 0) {
            const unsigned rowb = (unsigned)((nloc + 3) & ~3) * 4u;
            for (int c = 0; c < 3 * ND; ++c)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.q0lo + (size_t)c * P_ + e0),
                             "r"(rowb)
                             : "memory");
        }
    }
    int2 hrec = make_int2(0, -1);
    if (CAPPED && tid < nh) hrec = A.halo[hoff + tid];
    bool hwet = false;
    // stage increments: the halo staging holds q0f in its first 3 ND Real rows and d_s in the next 3 ND
    // (the same bytes as 3 ND doubles)
    Real* shf = reinterpret_cast<Real*>(shq);
    auto issue_halo_copies = [&]() {
        if constexpr (SPLIT) {
#pragma unroll
            for (int c = 0; c < 3 * ND; ++c) cp_async_value<Real>(&shf[c * max_halo + tid], &A.q0f[c * P_ + hrec.x]);
            if (A.dk[A.nterms - 1]) {
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c)
                    cp_async_value<Real>(&shf[(3 * ND + c) * max_halo + tid], &A.dk[A.nterms - 1][c * P_ + hrec.x]);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3 * ND; ++c) cp_async_value<double>(&shq[c * max_halo + tid], &qs[c * P_ + hrec.x]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) cp_async_value<Real>(&shb[k * max_halo + tid], &A.bath[k * P_ + hrec.x]);
        hwet = A.wet_in[hrec.x] != 0;
    };
    // an element's stage state in Real: q_s (FP64 stage states) or q0f + d_s (stage increments)
    auto load_state = [&](Real (&q)[3][ND], int e) {
        if constexpr (SPLIT) {
            const Real* __restrict__ ds = A.dk[A.nterms - 1];
            if (ds) {
                Real a[3 * ND], b[3 * ND];
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c) a[c] = A.q0f[c * P_ + e];
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c) b[c] = ds[c * P_ + e];
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = a[c] + b[c];
            } else {
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = A.q0f[c * P_ + e];
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = (Real)qs[c * P_ + e];
        }
    };

    // ---------------- phase 1: volume + source integrals, face traces ----------------
    if (active) {
        Real q[3][ND], b[3];
        load_state(q, d);
        if (CAPPED && hrec.y >= 0) issue_halo_copies();
#pragma unroll
        for (int k = 0; k < 3; ++k) b[k] = A.bath[k * P_ + d];
        const Real Ji00 = A.geo[d], Ji01 = A.geo[P_ + d], Ji10 = A.geo[2 * P_ + d], Ji11 = A.geo[3 * P_ + d];
        aJ = A.geo[4 * P_ + d];
        wet = A.wet_in[d] != 0;
        // the vertex coordinates (analytic source, spherical correction), loaded ahead of the wet test so that
        // the node-index and coordinate loads overlap the state loads instead of following the wet flag.
        // Measured per step on 524,288 triangles: FP32 p = 2 -1.3 to -1.9 %, p = 1 -3 to -4 % in both
        // precisions; FP64 p = 2, whose register budget is tightest, +2 to +3 %, so there they follow it.
        constexpr bool xy_early = sizeof(Real) == 4 || P == 1;
        double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0;
        auto load_xy = [&]() {
            if (FSRC || A.spherical) {
                const int n0 = A.enodes[d], n1 = A.enodes[P_ + d], n2 = A.enodes[2 * P_ + d];
                const double2 p0 = A.xy[n0], p1 = A.xy[n1], p2 = A.xy[n2];
                x0 = p0.x, y0 = p0.y, x1 = p1.x, y1 = p1.y, x2 = p2.x, y2 = p2.y;
            }
        };
        if constexpr (xy_early) load_xy();
        if (wet) {
            if constexpr (!xy_early) load_xy();
            // bathymetry gradient: the projected bathymetry is linear, its gradient constant
            Real db0 = Real(0), db1 = Real(0);
            sfor<0, 3>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr double c0 = MT<P>::dphi((0 * ND + k) * NQ + 0);
                constexpr double c1 = MT<P>::dphi((1 * ND + k) * NQ + 0);
                if constexpr (c0 != 0.0) db0 += b[k] * (Real)c0;
                if constexpr (c1 != 0.0) db1 += b[k] * (Real)c1;
            });
            const Real dbx = db0 * Ji00 + db1 * Ji10;
            const Real dby = db0 * Ji01 + db1 * Ji11;
            sfor<0, NQ>([&](auto GP) {
                constexpr int gp = decltype(GP)::value;
                Real qg[3];
                Real bg = Real(0);
                if constexpr (packed) {
                    // packed FP32: (ze, qx) and (qy, bathymetry) share each mode's coefficient
                    qg[0] = qg[1] = qg[2] = Real(0);
                    sfor<0, ND>([&](auto K) {
                        constexpr int k = decltype(K)::value;
                        constexpr double c = MT<P>::phi(k * NQ + gp);
                        if constexpr (c != 0.0) {
                            fma_pair(qg[0], qg[1], q[0][k], q[1][k], (Real)c, (Real)c);
                            if constexpr (k < 3)
                                fma_pair(qg[2], bg, q[2][k], b[k], (Real)c, (Real)c);
                            else
                                qg[2] = __fmaf_rn(q[2][k], (Real)c, qg[2]);
                        }
                    });
                } else {
                    sfor<0, 3>([&](auto V) {
                        constexpr int v = decltype(V)::value;
                        Real s = Real(0);
                        sfor<0, ND>([&](auto K) {
                            constexpr int k = decltype(K)::value;
                            constexpr double c = MT<P>::phi(k * NQ + gp);
                            if constexpr (c != 0.0) s += q[v][k] * (Real)c;
                        });
                        qg[v] = s;
                    });
                    sfor<0, 3>([&](auto K) {
                        constexpr int k = decltype(K)::value;
                        constexpr double c = MT<P>::phi(k * NQ + gp);
                        if constexpr (c != 0.0) bg += b[k] * (Real)c;
                    });
                }
                // physical flux, swe_flux.hpp:5-25
                const Real h = qg[0] + bg;
                const Real ih = Real(1) / h;
                const Real u = qg[1] * ih, vv = qg[2] * ih;
                const Real pe = g * (Real(0.5) * qg[0] * qg[0] + qg[0] * bg);
                Real Fx[3] = {qg[1], u * qg[1] + pe, u * qg[2]};
                Real Fy[3] = {qg[2], u * qg[2], vv * qg[2] + pe};
                double yg = 0.0;
                if (A.spherical) {
                    constexpr double s0 = MT<P>::psi(0 * NQ + gp), s1 = MT<P>::psi(1 * NQ + gp),
                                     s2 = MT<P>::psi(2 * NQ + gp);
                    yg = y0 * s0 + y1 * s1 + y2 * s2;
                }
                if (A.spherical) {
                    const Real sp = (Real)(A.sp_cos_lat0 / cos(yg / A.sp_R));
#pragma unroll
                    for (int v = 0; v < 3; ++v) Fx[v] = sp * Fx[v];
                }
                // bathymetry-slope source, swe_source.hpp:15-21 (the analytic source follows in its own loop,
                // except the manufactured sine set in FP32, added here: its sum then shares the phi w products)
                Real S[3] = {Real(0), g * (dbx * qg[0]), g * (dby * qg[0])};
                if constexpr (FSRC && sizeof(Real) == 4) {
                    if (sine_set) {
                        constexpr double s0 = MT<P>::psi(0 * NQ + gp), s1 = MT<P>::psi(1 * NQ + gp),
                                         s2 = MT<P>::psi(2 * NQ + gp);
                        const Real xg = (Real)x0 * (Real)s0 + (Real)x1 * (Real)s1 + (Real)x2 * (Real)s2;
                        const Real yg = (Real)y0 * (Real)s0 + (Real)y1 * (Real)s1 + (Real)y2 * (Real)s2;
                        Real fs[3];
                        sine_src_eval<Real>(SS, xg, yg, fs);
                        S[0] = fs[0];
                        S[1] += fs[1];
                        S[2] += fs[2];
                    }
                }
                // bottom friction, swe_source.hpp:29-51: S(qx, qy) -= Cf |u| / h (qx, qy), Cf the Chezy
                // coefficient or, for Manning, max(g n^2 / h^(1/3), Cf); |u| as sqrt(u^2 + v^2) and / h as
                // * (1 / h) where the reference has hypot and a division (each within an ulp; velocities
                // are far from hypot's overflow range)
                if (FRIC) {
                    const Real cf = A.friction == DGSW_FRICTION_MANNING ? manning_cf<Real>(A.manning[d], h, (Real)A.friction_cf)
                                                                        : (Real)A.friction_cf;
                    const Real tau = cf * sqrt(u * u + vv * vv) * ih;
                    S[1] -= tau * qg[1];
                    S[2] -= tau * qg[2];
                }
                // int F . grad(phi) = sum_gp sum_z (F_x J^-1(z,x) + F_y J^-1(z,y)) dphi_z w
                if constexpr (packed) {
                    // packed FP32: ze and qx share each mode's coefficients (qy alone), each mode's terms in the
                    // scalar loop's order
                    Real G0[3], G1[3];
#pragma unroll
                    for (int v = 0; v < 3; ++v) {
                        G0[v] = Fx[v] * Ji00 + Fy[v] * Ji01;
                        G1[v] = Fx[v] * Ji10 + Fy[v] * Ji11;
                    }
                    sfor<0, ND>([&](auto K) {
                        constexpr int k = decltype(K)::value;
                        constexpr double m0 = MT<P>::mz((0 * NQ + gp) * ND + k);
                        constexpr double m1 = MT<P>::mz((1 * NQ + gp) * ND + k);
                        constexpr double pw = MT<P>::phiw(gp * ND + k);
                        if constexpr (m0 != 0.0) {
                            fma_pair(rhs[0][k], rhs[1][k], G0[0], G0[1], (Real)m0, (Real)m0);
                            rhs[2][k] = __fmaf_rn(G0[2], (Real)m0, rhs[2][k]);
                        }
                        if constexpr (m1 != 0.0) {
                            fma_pair(rhs[0][k], rhs[1][k], G1[0], G1[1], (Real)m1, (Real)m1);
                            rhs[2][k] = __fmaf_rn(G1[2], (Real)m1, rhs[2][k]);
                        }
                        if constexpr (pw != 0.0) {
                            fma_pair(rhs[0][k], rhs[1][k], S[0], S[1], (Real)pw, (Real)pw);
                            rhs[2][k] = __fmaf_rn(S[2], (Real)pw, rhs[2][k]);
                        }
                    });
                    return;
                }
                sfor<0, 3>([&](auto V) {
                    constexpr int v = decltype(V)::value;
                    const Real G0 = Fx[v] * Ji00 + Fy[v] * Ji01;
                    const Real G1 = Fx[v] * Ji10 + Fy[v] * Ji11;
                    sfor<0, ND>([&](auto K) {
                        constexpr int k = decltype(K)::value;
                        constexpr double m0 = MT<P>::mz((0 * NQ + gp) * ND + k);
                        constexpr double m1 = MT<P>::mz((1 * NQ + gp) * ND + k);
                        constexpr double pw = MT<P>::phiw(gp * ND + k);
                        Real acc = rhs[v][k];
                        if constexpr (m0 != 0.0) acc += G0 * (Real)m0;
                        if constexpr (m1 != 0.0) acc += G1 * (Real)m1;
                        if constexpr (pw != 0.0) acc += S[v] * (Real)pw;
                        rhs[v][k] = acc;
                    });
                });
            });
            // analytic source_q(t, x_gp) (swe_source.hpp:9-14), in a loop of its own so that its
            // temporaries are not live together with the flux computation's
            // The manufactured sine set in FP64 on elements small against its wavelength (k times the
            // largest vertex offset from the centroid <= 0.05): sin and cos once at the centroid, turned to
            // each quadrature point by rotate_small; the point's offset from the centroid is
            // sum_i (psi_i - 1/3) (x_i - x_0), its coordinate never formed. Measured on 524,288 triangles at
            // p = 2: FP64 stage 212 -> 201 us; in FP32 the hardware sine/cosine per point stays cheaper
            // (114 against 116 us).
            const double xc = (x0 + x1 + x2) * (1.0 / 3.0), yc = (y0 + y1 + y2) * (1.0 / 3.0);
            bool near = false;
            if constexpr (sizeof(Real) == 8)
                near = sine_set && (double)SS.k * fmax(fmax(fmax(fabs(x0 - xc), fabs(x1 - xc)), fabs(x2 - xc)),
                                                         fmax(fmax(fabs(y0 - yc), fabs(y1 - yc)), fabs(y2 - yc))) <= 0.05;
            if constexpr (sizeof(Real) == 8) {
                if (FSRC && near) {
                    double sxc, cxc, syc, cyc;
                    sine_src_sincos<Real>(SS, xc, sxc, cxc);
                    sine_src_sincos<Real>(SS, yc, syc, cyc);
                    const double ex1 = x1 - x0, ex2 = x2 - x0, ey1 = y1 - y0, ey2 = y2 - y0;
                    sfor<0, NQ>([&](auto GP) {
                        constexpr int gp = decltype(GP)::value;
                        constexpr double a1 = MT<P>::psi(1 * NQ + gp) - 1.0 / 3.0, a2 = MT<P>::psi(2 * NQ + gp) - 1.0 / 3.0;
                        double sx, cx, sy, cy;
                        rotate_small(sxc, cxc, SS.k * (ex1 * a1 + ex2 * a2), sx, cx);
                        rotate_small(syc, cyc, SS.k * (ey1 * a1 + ey2 * a2), sy, cy);
                        Real fs[3];
                        sine_src_terms<Real>(SS, sx, cx, sy, cy, fs);
                        sfor<0, 3>([&](auto V) {
                            constexpr int v = decltype(V)::value;
                            sfor<0, ND>([&](auto K) {
                                constexpr int k = decltype(K)::value;
                                constexpr double pw = MT<P>::phiw(gp * ND + k);
                                if constexpr (pw != 0.0) rhs[v][k] += fs[v] * (Real)pw;
                            });
                        });
                    });
                }
            }
            if (FSRC && !near && !(sizeof(Real) == 4 && sine_set)) {
                const Real xr0 = (Real)x0, xr1 = (Real)x1, xr2 = (Real)x2;
                const Real yr0 = (Real)y0, yr1 = (Real)y1, yr2 = (Real)y2;
                sfor<0, NQ>([&](auto GP) {
                    constexpr int gp = decltype(GP)::value;
                    constexpr double s0 = MT<P>::psi(0 * NQ + gp), s1 = MT<P>::psi(1 * NQ + gp),
                                     s2 = MT<P>::psi(2 * NQ + gp);
                    // FP32 path: Gauss-point coordinates in FP32 (the analytic source is evaluated in FP32)
                    const Real xg = xr0 * (Real)s0 + xr1 * (Real)s1 + xr2 * (Real)s2;
                    const Real yg = yr0 * (Real)s0 + yr1 * (Real)s1 + yr2 * (Real)s2;
                    Real fs[3];
                    if (sine_set && sizeof(Real) == 8) {
                        // FP64 elements large against the wavelength: out of line, so that this rarely
                        // taken path keeps the kernel's hot code small
                        const Val3<Real> r = sine_src_far<Real>(A.fn_params, &FT, xg, yg);
                        fs[0] = r.v0, fs[1] = r.v1, fs[2] = r.v2;
                    } else if (sine_set) {
                        sine_src_eval<Real>(SS, xg, yg, fs);
                    } else {
                        const Val3<Real> r = fn_eval_dev<Real>(A.fn_set, A.fn_params, &FT, 1, xg, yg);
                        fs[0] = r.v0, fs[1] = r.v1, fs[2] = r.v2;
                    }
                    sfor<0, 3>([&](auto V) {
                        constexpr int v = decltype(V)::value;
                        sfor<0, ND>([&](auto K) {
                            constexpr int k = decltype(K)::value;
                            constexpr double pw = MT<P>::phiw(gp * ND + k);
                            if constexpr (pw != 0.0) rhs[v][k] += fs[v] * (Real)pw;
                        });
                    });
                });
            }
            // the volume integrals stay in master-element units: sol = (|J| V + E) M^-1 / |J| is
            // computed as V M^-1 + (E / |J|) M^-1, with 1 / |J| folded into the edge weights below
        }
        // traces of the three faces (needed also when dry: a wet neighbour evaluates the interface)
        sfor<0, 3>([&](auto FF) {
            constexpr int f = decltype(FF)::value;
            Real t[4][NG];
            face_trace<P, f, Real, packed>(q, b, t);
            const int slot = 3 * tid + f;
            put_trace(slot, t);
            swet[slot] = wet ? 1 : 0;
        });
    }
    // halo faces: faces of elements in other tiles that this tile's edges need
    if (CAPPED) {
        if (hrec.y >= 0) {
            if (!active) issue_halo_copies();  // threads past the last element of the last tile
            const int h = tid;
            cp_async_commit_and_wait();  // this thread's own copies
            Real q[3][ND], b[3], t[4][NG];
            if constexpr (SPLIT) {
                if (A.dk[A.nterms - 1]) {
#pragma unroll
                    for (int c = 0; c < 3 * ND; ++c)
                        q[c / ND][c % ND] = shf[c * max_halo + h] + shf[(3 * ND + c) * max_halo + h];
                } else {
#pragma unroll
                    for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = shf[c * max_halo + h];
                }
            } else {
#pragma unroll
                for (int c = 0; c < 3 * ND; ++c) q[c / ND][c % ND] = (Real)shq[c * max_halo + h];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) b[k] = shb[k * max_halo + h];
            if constexpr (rt_face) {
                face_trace_rt<P, Real, packed>(q, b, sfphi + hrec.y * ND * NG, t);
            } else if (hrec.y == 0) {
                face_trace<P, 0, Real, packed>(q, b, t);
            } else if (hrec.y == 1) {
                face_trace<P, 1, Real, packed>(q, b, t);
            } else {
                face_trace<P, 2, Real, packed>(q, b, t);
            }
            const int slot = 3 * TILE + h;
            put_trace(slot, t);
            swet[slot] = hwet ? 1 : 0;
        }
    } else {
#pragma unroll 1
        for (int h = tid; h < nh; h += TILE) {
            const int2 it = A.halo[hoff + h];
            const int e = it.x;
            Real q[3][ND], b[3], t[4][NG];
            load_state(q, e);
#pragma unroll
            for (int k = 0; k < 3; ++k) b[k] = A.bath[k * P_ + e];
            if constexpr (rt_face) {
                face_trace_rt<P, Real, packed>(q, b, sfphi + it.y * ND * NG, t);
            } else if (it.y == 0) {
                face_trace<P, 0, Real, packed>(q, b, t);
            } else if (it.y == 1) {
                face_trace<P, 1, Real, packed>(q, b, t);
            } else {
                face_trace<P, 2, Real, packed>(q, b, t);
            }
            const int slot = 3 * TILE + h;
            put_trace(slot, t);
            swet[slot] = A.wet_in[e] != 0 ? 1 : 0;
        }
    }
    // the first edge record and geometry of phase 2 are loaded before the barrier, so that their latency
    // overlaps the wait for the CTA's other warps (measured per step on 524,288-2,097,152 triangles: -0.6 to
    // -1.6 %; FP64 at p = 2, whose register budget is tightest, loads them after the barrier)
    constexpr bool edge_early = !(sizeof(Real) == 8 && P == 2);
    int4 rec_e = make_int4(0, 0, 0, 0);
    Real nx_e = Real(0), ny_e = Real(0), sj_e = Real(0);
    if (edge_early && tid < nedge) {
        rec_e = A.edges[eoff + tid];
        nx_e = A.egeo[eoff + tid];
        ny_e = A.egeo[A.n_edges + eoff + tid];
        sj_e = A.egeo[2 * A.n_edges + eoff + tid];
    }
    __syncthreads();

    // ---------------- phase 2: edge fluxes, once per edge of the tile ----------------
    {
        // the next edge's record and geometry are loaded one iteration ahead
        int4 rec_n = rec_e;
        Real nx_n = nx_e, ny_n = ny_e, sj_n = sj_e;
        if (!edge_early && tid < nedge) {
            rec_n = A.edges[eoff + tid];
            nx_n = A.egeo[eoff + tid];
            ny_n = A.egeo[A.n_edges + eoff + tid];
            sj_n = A.egeo[2 * A.n_edges + eoff + tid];
        }
#pragma unroll 1
        for (int le = tid; le < nedge; le += TILE) {
            const int4 rec = rec_n;
            const Real nx = nx_n, ny = ny_n;
            ssJ[le] = sj_n;
            if (le + TILE < nedge) {
                const int nle = eoff + le + TILE;
                rec_n = A.edges[nle];
                nx_n = A.egeo[nle];
                ny_n = A.egeo[A.n_edges + nle];
                sj_n = A.egeo[2 * A.n_edges + nle];
            }
            const int sa = rec.x, sb = rec.y;
            const int kind = (rec.z >> 4) & 7;
            const bool wa = swet[sa] != 0;
            const bool wb = sb >= 0 && swet[sb] != 0;
            const bool compute = (kind == 0 || kind == 5) ? (wa || wb) : wa;
            // 2 marks a levee interface: its ex-side flux is not -F and is read in phase 3
            sflag[le] = compute ? (kind == 5 ? 2 : 1) : 0;
            if (!compute) continue;
            if (kind == 5) {
                // the in-side flux as for any edge; the ex-side flux over the ex face's own trace slot,
                // which no other edge reads
                const double* Fl = A.levF + (size_t)(rec.z >> 8) * (6 * NG);
#pragma unroll
                for (int c = 0; c < 3 * NG; ++c) sF[c * max_edges + le] = (Real)Fl[c];
#pragma unroll
                for (int c = 0; c < 3 * NG; ++c) tr_at(c / NG, c % NG, sb) = (Real)Fl[3 * NG + c];
                continue;
            }
            Real sp = Real(1);
            double xa = 0, ya = 0, xb = 0, yb = 0;
            if (kind == 2 || A.spherical) {
                // Gauss points of face fa lie on the segment from node (fa+1)%3 to node (fa+2)%3
                const int fa = rec.z & 3, ea = rec.w;
                const double2 pa = A.xy[A.enodes[((fa + 1) % 3) * P_ + ea]];
                const double2 pb = A.xy[A.enodes[((fa + 2) % 3) * P_ + ea]];
                xa = pa.x, ya = pa.y, xb = pb.x, yb = pb.y;
            }
            sfor<0, NG>([&](auto GP) {
                constexpr int gp = decltype(GP)::value;
                constexpr int ge = NG - 1 - gp;  // the ex side's Gauss point paired with gp
                // BoundaryToMasterCoordinates + LocalToGlobalCoordinates on a straight edge
                constexpr double wa_ = MT<P>::fpsi((0 * 3 + 1) * NG + gp), wb_ = MT<P>::fpsi((0 * 3 + 2) * NG + gp);
                if (A.spherical) sp = (Real)(A.sp_cos_lat0 / cos((ya * wa_ + yb * wb_) / A.sp_R));
                Real qi[3], bi;
                if constexpr (tr_vec) {
                    const float4 a = *reinterpret_cast<const float4*>(str + (sa * NG + gp) * 4);
                    qi[0] = a.x, qi[1] = a.y, qi[2] = a.z, bi = a.w;
                } else {
                    qi[0] = str[(0 * NG + gp) * NS + sa], qi[1] = str[(1 * NG + gp) * NS + sa];
                    qi[2] = str[(2 * NG + gp) * NS + sa], bi = str[(3 * NG + gp) * NS + sa];
                }
                Real qe[3], be = Real(0);
                if (kind == 0) {
                    if constexpr (tr_vec) {
                        const float4 e = *reinterpret_cast<const float4*>(str + (sb * NG + ge) * 4);
                        qe[0] = e.x, qe[1] = e.y, qe[2] = e.z;
                        if (WD) be = e.w;
                    } else {
                        qe[0] = str[(0 * NG + ge) * NS + sb];
                        qe[1] = str[(1 * NG + ge) * NS + sb];
                        qe[2] = str[(2 * NG + ge) * NS + sb];
                        if (WD) be = str[(3 * NG + ge) * NS + sb];
                    }
                } else if (kind == 1) {
                    // BC::Land ghost state: normal momentum mirrored (rkdg_swe_bc_land.hpp:44-56)
                    const Real tx = -ny, ty = nx;
                    const Real qn_ex = -(qi[1] * nx + qi[2] * ny);
                    const Real qt_ex = qi[1] * tx + qi[2] * ty;
                    qe[0] = qi[0];
                    qe[1] = qn_ex * nx + qt_ex * tx;
                    qe[2] = qn_ex * ny + qt_ex * ty;
                } else {
                    // function, tide and flow boundaries (a tide / flow face's b slot holds -2 - its
                    // forcing record)
                    const Val3<Real> r =
                        boundary_ghost<Real>(&A, &FT, kind, -2 - sb, gp, t_stage, (Real)(xa * wa_ + xb * wb_),
                                             (Real)(ya * wa_ + yb * wb_), qi[0], qi[1], qi[2], nx, ny);
                    qe[0] = r.v0, qe[1] = r.v1, qe[2] = r.v2;
                }
                Real Fi[3];
                // packed at p = 1 only: measured per step, the p = 1 tidal channel -1.7 %; at p = 2 the kernel
                // spilled and the config-2 step took 2 % longer
                if constexpr (packed && P == 1)
                    llf_flux_packed(g, qi, qe, bi, sp, nx, ny, Fi);
                else
                    llf_flux<Real>(g, qi, qe, bi, sp, nx, ny, Fi);
                if (WD && kind == 0) {
                    Real Fe[3] = {-Fi[0], -Fi[1], -Fi[2]};
                    if (!(wa && wb)) {
                        const Flux2<Real> r = wd_fixup<Real>(g, qi[0], qi[1], qi[2], qe[0], qe[1], qe[2], bi, be, sp,
                                                             nx, ny, wa, wb, Fi[0], Fi[1], Fi[2]);
                        Fi[0] = r.i0, Fi[1] = r.i1, Fi[2] = r.i2;
                        Fe[0] = r.e0, Fe[1] = r.e1, Fe[2] = r.e2;
                    }
#pragma unroll
                    for (int v = 0; v < 3; ++v) sF[((3 + v) * NG + gp) * max_edges + le] = Fe[v];
                }
#pragma unroll
                for (int v = 0; v < 3; ++v) sF[(v * NG + gp) * max_edges + le] = Fi[v];
            });
        }
    }
    double comb[3][ND];
    double bv[3] = {0.0, 0.0, 0.0};
    // phase 3's global loads: the RK combination's state terms and the wet/dry vertex depths, issued when
    // phase 3 starts (issuing them before the CTA's second barrier instead gained nothing, measured on the
    // p = 1 and p = 2 workloads in both precisions)
    auto load_phase3 = [&]() {
        if constexpr (SPLIT) split_comb();
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < ND; ++k) comb[v][k] = 0.0;
        for (int j = 0; j < (SPLIT ? 0 : A.nterms); ++j) {
            const double* __restrict__ qj = A.qk[j];
            const double aj = A.a[j];
            double t[3][ND];
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) t[v][k] = qj[(v * ND + k) * P_ + d];
            if (j < A.nterms - 1 && A.bdt[j] != 0.0) {
                const double* __restrict__ sj = A.solk[j];
                const double bj = A.bdt[j];
                double u[3][ND];
#pragma unroll
                for (int v = 0; v < 3; ++v)
#pragma unroll
                    for (int k = 0; k < ND; ++k) u[v][k] = sj[(v * ND + k) * P_ + d];
#pragma unroll
                for (int v = 0; v < 3; ++v)
#pragma unroll
                    for (int k = 0; k < ND; ++k) comb[v][k] += bj * u[v][k];
            }
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) comb[v][k] += aj * t[v][k];
        }
        // wetting/drying: the element's vertex depths, loaded now (two dependent loads) so that their latency
        // overlaps the edge gather instead of opening the wet/dry pass
        if (WD) {
            const int n0 = A.enodes[d], n1 = A.enodes[P_ + d], n2 = A.enodes[2 * P_ + d];
            bv[0] = A.nz[n0], bv[1] = A.nz[n1], bv[2] = A.nz[n2];
        }
    };
    __syncthreads();

    // ---------------- phase 3: edge contributions, M^-1, RK combination, wet/dry ----------------
    if (!active) return;
    // the RK combination's state terms, sum_j a_j q_j + dt b_j sol_j over the earlier stages plus
    // a_s q_s, in FP64: all loads of one term are issued together here so that their latency overlaps
    // the edge gather below (one dependent load per value at the end of the CTA cost a global-memory
    // latency per value, per wave)
    load_phase3();
    const Real iaJ = Real(1) / aJ;
    const int roles = es.y & 7;
    const int ord = es.y >> 3;
    const int cnt = ord & 3;
#pragma unroll 1
    for (int i = 0; i < cnt; ++i) {
        const int f = (ord >> (2 + 2 * i)) & 3;
        const int slot = (es.x >> (10 * f)) & 1023;
        const int sfl = sflag[slot];
        if (!sfl) continue;
        const bool is_in = (roles >> f) & 1;
        const Real sJe = ssJ[slot] * iaJ;  // edge half length over |J|
        Real F[3][NG];
#pragma unroll
        for (int gp = 0; gp < NG; ++gp) {  // own Gauss point order
            if (is_in) {
#pragma unroll
                for (int v = 0; v < 3; ++v) F[v][gp] = sF[(v * NG + gp) * max_edges + slot];
            } else if (sfl == 2) {  // levee ex side: its own flux, left in its face's trace slot
#pragma unroll
                for (int v = 0; v < 3; ++v) F[v][gp] = tr_at(v, NG - 1 - gp, 3 * tid + f);
            } else {
                const int ga = NG - 1 - gp;
#pragma unroll
                for (int v = 0; v < 3; ++v)
                    F[v][gp] = WD ? sF[((3 + v) * NG + ga) * max_edges + slot] : -sF[(v * NG + ga) * max_edges + slot];
            }
        }
        if constexpr (rt_face) {
            // rhs -= sum_gp F phi_k w |e|/2 / |J| with the face's basis values from shared memory (a value
            // that is zero on this face but not on another subtracts a zero product: the sum is unchanged)
            const Real* __restrict__ cf = sfphi + f * ND * NG;
            sfor<0, NG>([&](auto GP) {
                constexpr int gp = decltype(GP)::value;
                const Real wsJ = (Real)MT<P>::gw(gp) * sJe;
                Real T[3];
#pragma unroll
                for (int v = 0; v < 3; ++v) T[v] = F[v][gp] * wsJ;
                sfor<0, ND>([&](auto K) {
                    constexpr int k = decltype(K)::value;
                    constexpr bool used = MT<P>::fphi((0 * ND + k) * NG + gp) != 0.0 ||
                                          MT<P>::fphi((1 * ND + k) * NG + gp) != 0.0 ||
                                          MT<P>::fphi((2 * ND + k) * NG + gp) != 0.0;
                    if constexpr (used) {
                        const Real c = cf[k * NG + gp];
                        if constexpr (packed) {
                            // packed FP32: ze and qx share the coefficient (qy alone), as fma(-T, c, rhs)
                            fma_pair(rhs[0][k], rhs[1][k], -T[0], -T[1], c, c);
                            rhs[2][k] = __fmaf_rn(-T[2], c, rhs[2][k]);
                        } else {
#pragma unroll
                            for (int v = 0; v < 3; ++v) rhs[v][k] -= T[v] * c;
                        }
                    }
                });
            });
        } else {
            auto contrib = [&](auto FF) {
                constexpr int fc = decltype(FF)::value;
                sfor<0, NG>([&](auto GP) {
                    constexpr int gp = decltype(GP)::value;
                    const Real wsJ = (Real)MT<P>::gw(gp) * sJe;
                    Real T[3];
#pragma unroll
                    for (int v = 0; v < 3; ++v) T[v] = F[v][gp] * wsJ;
                    sfor<0, ND>([&](auto K) {
                        constexpr int k = decltype(K)::value;
                        constexpr double c = MT<P>::fphi((fc * ND + k) * NG + gp);
                        if constexpr (c != 0.0) {
                            if constexpr (packed) {
                                // packed FP32: ze and qx share the coefficient (qy alone), as fma(-T, c, rhs)
                                fma_pair(rhs[0][k], rhs[1][k], -T[0], -T[1], (Real)c, (Real)c);
                                rhs[2][k] = __fmaf_rn(-T[2], (Real)c, rhs[2][k]);
                            } else {
#pragma unroll
                                for (int v = 0; v < 3; ++v) rhs[v][k] -= T[v] * (Real)c;
                            }
                        }
                    });
                });
            };
            if (f == 0)
                contrib(IC<0>{});
            else if (f == 1)
                contrib(IC<1>{});
            else
                contrib(IC<2>{});
        }
    }
    // M^-1 (the diagonal master mass inverse; 1 / |J| is already in) and the SSP-RK stage combination
    const double bdt_s = A.bdt[A.nterms - 1];
    if constexpr (SPLIT) {
        const Real bs = (Real)bdt_s;
        // dn = dcomb + dt b_s (rhs M^-1), ze and qx packed (each lane the scalar mul and fma)
        Real (&dn)[3][ND] = dcomb;
        sfor<0, ND>([&](auto K) {
            constexpr int k = decltype(K)::value;
            const Real mk = (Real)MT<P>::minv(k);
            const float2 s01 = __fmul2_rn(make_float2(rhs[0][k], rhs[1][k]), make_float2(mk, mk));
            const Real sol[3] = {s01.x, s01.y, rhs[2][k] * mk};
            if (A.store_sol) {
#pragma unroll
                for (int v = 0; v < 3; ++v) A.dsol_out[(v * ND + k) * P_ + d] = sol[v];
            }
            fma_pair(dn[0][k], dn[1][k], sol[0], sol[1], bs, bs);
            dn[2][k] = __fmaf_rn(sol[2], bs, dn[2][k]);
        });
        bool has_nan = false;
        if (A.last) {
            // the new carried state q0f + q0lo + d_ns in FP64 (q0f + q0lo is exact there), split again into
            // its leading and trailing Real parts; q_0 is loaded here rather than with the increments (held
            // across the edge gather its registers would spill; its leading part is an L1 or L2 hit from
            // phase 1)
            Real hi[3][ND], lo[3][ND];
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    hi[v][k] = A.q0f[(v * ND + k) * P_ + d];
                    lo[v][k] = A.q0lo[(v * ND + k) * P_ + d];
                }
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    const int idx = (v * ND + k) * P_ + d;
                    const double qv = ((double)hi[v][k] + (double)lo[v][k]) + (double)dn[v][k];
                    has_nan |= isnan(qv);
                    const Real h2 = (Real)qv;
                    A.q0f_out[idx] = h2;
                    A.q0lo_out[idx] = (Real)(qv - (double)h2);
                }
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    has_nan |= isnan(dn[v][k]);
                    A.d_out[(v * ND + k) * P_ + d] = dn[v][k];
                }
        }
        A.wet_out[d] = wet ? 1 : 0;
        if (has_nan) {
            const unsigned long long counter = (unsigned long long)A.clock->step * A.nstages + A.stage_index;
            atomicOr(&A.status->nan_flag, 1u);
            atomicMin(&A.status->nan_key, (counter << 32) | (unsigned int)A.ref_of_dev[d]);
        }
        return;
    }
    double qn[3][ND];
    sfor<0, ND>([&](auto K) {
        constexpr int k = decltype(K)::value;
        const Real mk = (Real)MT<P>::minv(k);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double sol = (double)(rhs[v][k] * mk);
            const int idx = (v * ND + k) * P_ + d;
            if (A.store_sol) A.sol_out[idx] = sol;
            qn[v][k] = comb[v][k] + bdt_s * sol;
        }
    });
    bool wet_new = wet;
    if (WD) {
        const double bmin = fmin(bv[0], fmin(bv[1], bv[2]));
        bool went_dry = false;
        wet_new = wetting_drying<ND, double>(qn, bv, bmin, A.h_o, A.h_o_thr, wet, went_dry);
        if (A.went_dry) A.went_dry[d] = went_dry ? 1 : 0;
    }
    bool has_nan = false;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            has_nan |= isnan((double)qn[v][k]);
            A.q_out[(v * ND + k) * P_ + d] = qn[v][k];
        }
    A.wet_out[d] = wet_new ? 1 : 0;
    if (A.baryctr) {
        // slope_limiting_prepare_element_kernel (swe_CS_slope_limiter.hpp:9-20): vertex values through
        // T_basis_linear, barycentre value = vertex values . (1/3, 1/3, 1/3)
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double a = qn[v][0], b = qn[v][1], c = qn[v][2];
            const double l0 = a - b - c, l1 = a - b + c, l2 = a + 2.0 * b;
            A.baryctr[v * P_ + d] = l0 * (1.0 / 3.0) + l1 * (1.0 / 3.0) + l2 * (1.0 / 3.0);
        }
    }
    if (has_nan) {
        const unsigned long long counter = (unsigned long long)A.clock->step * A.nstages + A.stage_index;
        atomicOr(&A.status->nan_flag, 1u);
        atomicMin(&A.status->nan_key, (counter << 32) | (unsigned int)A.ref_of_dev[d]);
    }
}

// launchers, one translation unit per (order, precision, register budget); bit 3 of `mode` selects the
// alternative budget (OCC = 1)
constexpr int STAGE_MODE_OCC = 8;
// bit 4 of `mode`: the kernel with run-time shared-memory strides even where the mesh fits the caps
constexpr int STAGE_MODE_UNCAPPED = 16;
cudaError_t launch_stage_p1_f64(const StageArgs<double>& A, int tile, int ntiles, int max_halo, int max_edges,
                                int mode, cudaStream_t s);
cudaError_t launch_stage_p1_f32(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                int mode, cudaStream_t s);
cudaError_t launch_stage_p2_f64(const StageArgs<double>& A, int tile, int ntiles, int max_halo, int max_edges,
                                int mode, cudaStream_t s);
cudaError_t launch_stage_p2_f32(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                int mode, cudaStream_t s);
cudaError_t launch_stage_p1_f64_occ(const StageArgs<double>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s);
cudaError_t launch_stage_p1_f32_occ(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s);
cudaError_t launch_stage_p2_f64_occ(const StageArgs<double>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s);
cudaError_t launch_stage_p2_f32_occ(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                    int mode, cudaStream_t s);
// stage increments (StageArgs::dk ...): the default budget, or the alternative one with bit 3 of `mode`
cudaError_t launch_stage_p1_f32_split(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                      int mode, cudaStream_t s);
cudaError_t launch_stage_p2_f32_split(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                      int mode, cudaStream_t s);

// whether every tile of a mesh fits the compile-time shared-memory capacities of the capped kernels
inline bool stage_fits_caps(int tile, int max_halo, int max_edges) {
    return tile == 128 ? max_halo <= TileCap<128>::halo && max_edges <= TileCap<128>::edges
                       : max_halo <= TileCap<256>::halo && max_edges <= TileCap<256>::edges;
}

// with `allow_capped` false the kernel with run-time strides runs even where the mesh fits the caps: its
// shared memory is sized to the mesh's largest tile, and with less shared memory per SM the L1 cache that
// shares its storage is larger (the autotuner times both)
template <int P, typename Real, bool WD, bool FSRC, bool FRIC, int TILE, int OCC, bool SPLIT = false>
cudaError_t launch_stage_impl(const StageArgs<Real>& A, int ntiles, int max_halo, int max_edges, bool allow_capped,
                              cudaStream_t s) {
    const bool capped = allow_capped && max_halo <= TileCap<TILE>::halo && max_edges <= TileCap<TILE>::edges;
    auto kern = capped ? rkdg_stage_kernel<P, Real, WD, FSRC, FRIC, TILE, true, OCC, SPLIT>
                       : rkdg_stage_kernel<P, Real, WD, FSRC, FRIC, TILE, false, OCC, SPLIT>;
    // the run-time-stride kernel loads its halo faces' elements straight from global memory and never
    // touches the halo staging area (every use of it is under CAPPED), so its allocation ends there
    const size_t smem = capped ? Smem<P, Real, WD>::bytes(TILE, TileCap<TILE>::halo, TileCap<TILE>::edges)
                               : Smem<P, Real, WD>::off_halo(TILE, max_halo, max_edges);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)ntiles, TILE, smem, s>>>(A, max_halo, max_edges);
    return cudaGetLastError();
}

template <int P, typename Real, bool WD, bool FSRC, bool FRIC, int OCC, bool SPLIT = false>
cudaError_t launch_stage_tile(const StageArgs<Real>& A, int tile, int ntiles, int max_halo, int max_edges, int mode,
                              cudaStream_t s) {
    const bool allow_capped = !(mode & STAGE_MODE_UNCAPPED);
    switch (tile) {
        case 128:
            return launch_stage_impl<P, Real, WD, FSRC, FRIC, 128, OCC, SPLIT>(A, ntiles, max_halo, max_edges,
                                                                                allow_capped, s);
        case 256:
            return launch_stage_impl<P, Real, WD, FSRC, FRIC, 256, OCC, SPLIT>(A, ntiles, max_halo, max_edges,
                                                                                allow_capped, s);
        default:
            return cudaErrorInvalidValue;
    }
}

// wetting/drying, function source and bottom friction select the instantiation (bit 0, 1, 2 of `mode`)
template <int P, typename Real, int OCC>
cudaError_t launch_stage_dispatch(const StageArgs<Real>& A, int tile, int ntiles, int max_halo, int max_edges,
                                  int mode, cudaStream_t s) {
    switch (mode & 7) {
        case 0: return launch_stage_tile<P, Real, false, false, false, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 1: return launch_stage_tile<P, Real, true, false, false, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 2: return launch_stage_tile<P, Real, false, true, false, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 3: return launch_stage_tile<P, Real, true, true, false, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 4: return launch_stage_tile<P, Real, false, false, true, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 5: return launch_stage_tile<P, Real, true, false, true, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 6: return launch_stage_tile<P, Real, false, true, true, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
        default: return launch_stage_tile<P, Real, true, true, true, OCC>(A, tile, ntiles, max_halo, max_edges, mode, s);
    }
}

// the stage-increment kernels (FP32, no wetting/drying): function source and bottom friction select the
// instantiation (bits 1 and 2 of `mode`; bit 0, wetting/drying, must be clear)
template <int P, int OCC>
cudaError_t launch_stage_split_dispatch(const StageArgs<float>& A, int tile, int ntiles, int max_halo, int max_edges,
                                        int mode, cudaStream_t s) {
    switch (mode & 7) {
        case 0: return launch_stage_tile<P, float, false, false, false, OCC, true>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 2: return launch_stage_tile<P, float, false, true, false, OCC, true>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 4: return launch_stage_tile<P, float, false, false, true, OCC, true>(A, tile, ntiles, max_halo, max_edges, mode, s);
        case 6: return launch_stage_tile<P, float, false, true, true, OCC, true>(A, tile, ntiles, max_halo, max_edges, mode, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace dgsw

#endif
