// CPU FP64 oracle for the dgswemv2 RKDG step. TEST INFRASTRUCTURE ONLY (see oracle.hpp).
//
// Each block cites the reference file:line it restates. The reference evaluates small dense
// products through Eigen expression templates; here every product is a plain loop that sums over
// the inner index in ascending order, and chained products are evaluated left to right.
#include "oracle.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../dgswemv2_b200/csrc/function_sets.h"
#include "../dgswemv2_b200/csrc/quadrature.h"
#include "../dgswemv2_b200/csrc/rk_tables.h"

namespace {

using std::vector;
thread_local std::string g_err;

constexpr uint32_t DEFAULT_ID = 4294967295u;  // general_definitions.hpp:230
constexpr int BT_LAND = 0, BT_TIDE = 1, BT_FLOW = 2, BT_FUNCTION = 3, BT_OUTFLOW = 4, BT_LEVEE = 129;
constexpr int BT_INTERNAL = 128;  // utilities/edge_types.hpp:4
constexpr double DBL_EPS = 2.220446049250313e-16;
constexpr double REF_PI = 3.14159265359;  // the reference's PI (general_definitions.hpp:227)

// ------------------------------------------------------------------------------------------------
// Jacobi polynomials, source/basis/polynomials/basis_polynomials.cpp:4-67
// ------------------------------------------------------------------------------------------------
double jacobi_polynomial(unsigned n, unsigned a, unsigned b, double x) {
    if (n == 0) return 1;
    if (n == 1) return (a - b + (a + b + 2) * x) / 2;
    double J[3];
    J[0] = 1.0;
    J[1] = (a - b + (a + b + 2) * x) / 2;
    J[2] = 0.0;
    for (unsigned i = 1; i < n; ++i) {
        double a1 = 2 * (i + 1) * (i + a + b + 1) * (2 * i + a + b);
        double a2 = (2 * i + a + b + 1) * (a * a - b * b);
        double a3 = (2 * i + a + b) * (2 * i + a + b + 1) * (2 * i + a + b + 2);
        double a4 = 2 * (i + a) * (i + b) * (2 * i + a + b + 2);
        J[(i + 1) % 3] = ((a2 + a3 * x) * J[i % 3] - a4 * J[(i - 1) % 3]) / a1;
    }
    return J[n % 3];
}

double jacobi_polynomial_derivative(unsigned n, unsigned a, unsigned b, double x) {
    if (n == 0) return 0.0;
    if (n == 1) return (a + b + n + 1) / 2.0;
    return jacobi_polynomial(n - 1, a + 1, b + 1, x) * ((a + b + n + 1) / 2.0);
}

// ------------------------------------------------------------------------------------------------
// Dubiner basis, source/basis/bases_2D/basis_dubiner_2D.cpp:4-211
// ------------------------------------------------------------------------------------------------
void dof_to_pq(unsigned dof, unsigned& p, unsigned& q) {
    unsigned tri_num_indx = (unsigned)std::ceil((-3. + std::sqrt(1. + 8. * (dof + 1))) / 2.);
    unsigned lower_tri_num = (tri_num_indx + 1) * tri_num_indx / 2;
    p = dof - lower_tri_num;
    q = tri_num_indx - p;
}

void singular_dz1(unsigned q, double out[2]) {  // :177-193
    if (q == 0) {
        out[0] = 3.;
        out[1] = 1.;
    } else {
        double t[2];
        singular_dz1(q - 1, t);
        out[0] = t[0] + q + 2;
        out[1] = t[0] + t[1];
    }
}

void singular_dz2(unsigned q, double out[2]) {  // :195-211
    if (q == 0) {
        out[0] = 0.5;
        out[1] = 0;
    } else {
        double t[2];
        singular_dz2(q - 1, t);
        out[0] = t[0] + 0.5 * (q + 1);
        out[1] = t[0] + t[1];
    }
}

double dubiner_phi(unsigned p, unsigned q, double z1, double z2) {  // :85-111
    double n1 = 2 * (1 + z1) / (1 - z2) - 1;
    double n2 = z2;
    double phi = jacobi_polynomial(p, 0, 0, n1) * std::pow((1 - n2) / 2, (int)p) * jacobi_polynomial(q, 2 * p + 1, 0, n2);
    if (std::isnan(n1)) phi = (p == 0) ? (double)(q + 1) : 0.0;
    return phi;
}

double dubiner_dphi_dz1(unsigned p, unsigned q, double z1, double z2) {  // :113-139
    double n1 = 2 * (1 + z1) / (1 - z2) - 1;
    double n2 = z2;
    double psi_pq = jacobi_polynomial(q, 2 * p + 1, 0, n2);
    double dpsi_p = jacobi_polynomial_derivative(p, 0, 0, n1);
    double v = (2.0 / (1.0 - n2)) * dpsi_p * std::pow((1.0 - n2) / 2.0, (int)p) * psi_pq;
    if (std::isnan(n1)) {
        if (p == 1) {
            double s[2];
            singular_dz1(q, s);
            v = s[1];
        } else {
            v = 0.0;
        }
    }
    return v;
}

double dubiner_dphi_dz2(unsigned p, unsigned q, double z1, double z2) {  // :141-175
    double n1 = 2 * (1 + z1) / (1 - z2) - 1;
    double n2 = z2;
    double psi_p = jacobi_polynomial(p, 0, 0, n1);
    double psi_pq = jacobi_polynomial(q, 2 * p + 1, 0, n2);
    double dpsi_p = jacobi_polynomial_derivative(p, 0, 0, n1);
    double dpsi_pq = jacobi_polynomial_derivative(q, 2 * p + 1, 0, n2);
    double v = ((1 + n1) / (1.0 - n2)) * dpsi_p * std::pow((1.0 - n2) / 2.0, (int)p) * psi_pq +
               psi_p * (std::pow((1.0 - n2) / 2.0, (int)p) * dpsi_pq -
                        (p / 2.0) * std::pow((1.0 - n2) / 2.0, (int)(p - 1)) * psi_pq);
    if (std::isnan(n1)) {
        double s[2];
        if (p == 0) {
            singular_dz2(q, s);
            v = 3 * s[1];
        } else if (p == 1) {
            singular_dz2(q + 1, s);
            v = s[1];
        } else {
            v = 0.0;
        }
    }
    return v;
}

// phi[dof*npt + pt]
vector<double> get_phi(int p, const vector<double>& z1, const vector<double>& z2) {
    int nd = (p + 1) * (p + 2) / 2, np = (int)z1.size();
    vector<double> phi(nd * np);
    for (int dof = 0; dof < nd; ++dof) {
        unsigned pp, qq;
        dof_to_pq(dof, pp, qq);
        for (int pt = 0; pt < np; ++pt) phi[dof * np + pt] = dubiner_phi(pp, qq, z1[pt], z2[pt]);
    }
    return phi;
}

void get_dphi(int p, const vector<double>& z1, const vector<double>& z2, vector<double>& d1, vector<double>& d2) {
    int nd = (p + 1) * (p + 2) / 2, np = (int)z1.size();
    d1.assign(nd * np, 0.0);
    d2.assign(nd * np, 0.0);
    for (int dof = 0; dof < nd; ++dof) {
        unsigned pp, qq;
        dof_to_pq(dof, pp, qq);
        for (int pt = 0; pt < np; ++pt) {
            d1[dof * np + pt] = dubiner_dphi_dz1(pp, qq, z1[pt], z2[pt]);
            d2[dof * np + pt] = dubiner_dphi_dz2(pp, qq, z1[pt], z2[pt]);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Master triangle, source/master/elements_2D/master_triangle.tpp:4-122
// ------------------------------------------------------------------------------------------------
struct Master {
    int p, nd, ngp;
    dgsw::Rule2D rule;
    vector<double> phi, dphi[2];          // [dof*ngp+gp]
    vector<double> int_phi, int_dphi[2];  // [gp*nd+dof]
    vector<double> minv;                  // diagonal
    double Tbl[6 * 3];                    // T_basis_linear (nd x 3), rows >= 3 zero (uses first 3 dofs)
    double Tlb[3 * 6];                    // T_linear_basis (3 x nd), only p >= 1 columns 0..2 nonzero
    double chi_baryctr[3];
    double chi_midpts[3][3];  // (vrtx, bound)

    void init(int p_) {
        p = p_;
        nd = (p + 1) * (p + 2) / 2;
        rule = dgsw::triangle_rule(2 * p);
        ngp = (int)rule.w.size();
        phi = get_phi(p, rule.z1, rule.z2);
        get_dphi(p, rule.z1, rule.z2, dphi[0], dphi[1]);
        int_phi.assign(ngp * nd, 0.0);
        for (int d = 0; d < 2; ++d) int_dphi[d].assign(ngp * nd, 0.0);
        for (int dof = 0; dof < nd; ++dof)
            for (int gp = 0; gp < ngp; ++gp) {
                int_phi[gp * nd + dof] = phi[dof * ngp + gp] * rule.w[gp];
                for (int d = 0; d < 2; ++d) int_dphi[d][gp * nd + dof] = dphi[d][dof * ngp + gp] * rule.w[gp];
            }
        minv.assign(nd, 0.0);
        for (int dof = 0; dof < nd; ++dof) {  // basis_dubiner_2D.cpp:65-83
            unsigned pp, qq;
            dof_to_pq(dof, pp, qq);
            minv[dof] = ((2 * pp + 1) * (pp + qq + 1) / 2.0);
        }
        // basis_dubiner_2D.cpp:213-257
        std::memset(Tbl, 0, sizeof(Tbl));
        std::memset(Tlb, 0, sizeof(Tlb));
        auto TBL = [&](int r, int c) -> double& { return Tbl[r * 3 + c]; };
        auto TLB = [&](int r, int c) -> double& { return Tlb[r * 6 + c]; };
        TBL(0, 0) = 1.0;
        TBL(1, 0) = -1.0;
        TBL(2, 0) = -1.0;
        TBL(0, 1) = 1.0;
        TBL(1, 1) = -1.0;
        TBL(2, 1) = 1.0;
        TBL(0, 2) = 1.0;
        TBL(1, 2) = 2.0;
        TBL(2, 2) = 0.0;
        TLB(0, 0) = 1.0 / 3.0;
        TLB(1, 0) = 1.0 / 3.0;
        TLB(2, 0) = 1.0 / 3.0;
        TLB(0, 1) = -1.0 / 6.0;
        TLB(1, 1) = -1.0 / 6.0;
        TLB(2, 1) = 1.0 / 3.0;
        TLB(0, 2) = -1.0 / 2.0;
        TLB(1, 2) = 1.0 / 2.0;
        TLB(2, 2) = 0.0;
        for (int i = 0; i < 3; ++i) chi_baryctr[i] = 1.0 / 3.0;
        double cm[3][3] = {{0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0}};
        std::memcpy(chi_midpts, cm, sizeof(cm));
    }

    // q_lin(var, vrtx) = sum_dof q(var,dof) T_basis_linear(dof, vrtx); q is [var*nd+dof]
    void basis_to_linear(const double* q, double ql[3][3]) const {
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < 3; ++k) {
                double s = 0.0;
                for (int dof = 0; dof < nd; ++dof) s += q[v * nd + dof] * (dof < 3 ? Tbl[dof * 3 + k] : 0.0);
                ql[v][k] = s;
            }
    }
    // q(var, dof) = sum_vrtx ql(var, vrtx) T_linear_basis(vrtx, dof)
    void linear_to_basis_row(const double ql[3], double* qrow) const {
        for (int dof = 0; dof < nd; ++dof) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += ql[k] * (dof < 3 ? Tlb[k * 6 + dof] : 0.0);
            qrow[dof] = s;
        }
    }
};

// boundary -> master coordinates, master_triangle.tpp:89-122
void bound_to_master(int bound_id, double z, double& z1, double& z2) {
    if (bound_id == 0) {
        z1 = -z;
        z2 = z;
    } else if (bound_id == 1) {
        z1 = -1.0;
        z2 = -z;
    } else {
        z1 = z;
        z2 = -1.0;
    }
}

// ------------------------------------------------------------------------------------------------
// Straight triangle shape, source/shape/shapes_2D/shape_straighttriangle.cpp
// ------------------------------------------------------------------------------------------------
struct Shape {
    double X[3][3];  // nodal coordinates (x, y, z)
    void J(double M[2][2]) const {
        M[0][0] = (X[1][0] - X[0][0]) / 2.0;
        M[0][1] = (X[2][0] - X[0][0]) / 2.0;
        M[1][0] = (X[1][1] - X[0][1]) / 2.0;
        M[1][1] = (X[2][1] - X[0][1]) / 2.0;
    }
    double detJ() const {
        double M[2][2];
        J(M);
        return M[0][0] * M[1][1] - M[1][0] * M[0][1];
    }
    void Jinv(double I[2][2]) const {  // 2x2 cofactor inverse
        double M[2][2];
        J(M);
        double invdet = 1.0 / (M[0][0] * M[1][1] - M[1][0] * M[0][1]);
        I[0][0] = M[1][1] * invdet;
        I[1][0] = -M[1][0] * invdet;
        I[0][1] = -M[0][1] * invdet;
        I[1][1] = M[0][0] * invdet;
    }
    double surface_J(int b) const {  // :110-122
        return std::sqrt(std::pow(X[(b + 2) % 3][0] - X[(b + 1) % 3][0], 2.0) +
                         std::pow(X[(b + 2) % 3][1] - X[(b + 1) % 3][1], 2.0)) /
               2.0;
    }
    void normal(int b, double n[2]) const {  // :139-168
        double det = detJ();
        double cw = det / std::abs(det);
        double length = std::hypot(X[(b + 2) % 3][0] - X[(b + 1) % 3][0], X[(b + 2) % 3][1] - X[(b + 1) % 3][1]);
        n[0] = cw * (X[(b + 2) % 3][1] - X[(b + 1) % 3][1]) / length;
        n[1] = -cw * (X[(b + 2) % 3][0] - X[(b + 1) % 3][0]) / length;
    }
    static void psi(double z1, double z2, double ps[3]) {  // :170-183
        ps[0] = -(z1 + z2) / 2;
        ps[1] = (1 + z1) / 2;
        ps[2] = (1 + z2) / 2;
    }
    void local_to_global(double z1, double z2, double& x, double& y) const {  // :229-247
        double ps[3];
        psi(z1, z2, ps);
        x = X[0][0] * ps[0] + X[1][0] * ps[1] + X[2][0] * ps[2];
        y = X[0][1] * ps[0] + X[1][1] * ps[1] + X[2][1] * ps[2];
    }
    double area() const {
        return 0.5 * (X[0][0] * (X[1][1] - X[2][1]) + X[1][0] * (X[2][1] - X[0][1]) + X[2][0] * (X[0][1] - X[1][1]));
    }
    double radius() const {
        double ret = 1.0 / (4 * area());
        for (int s = 0; s < 3; ++s) ret *= std::hypot(X[s][0] - X[(s + 1) % 3][0], X[s][1] - X[(s + 1) % 3][1]);
        return ret;
    }
    double length(int s) const {
        return std::hypot(X[(s + 1) % 3][0] - X[(s + 2) % 3][0], X[(s + 1) % 3][1] - X[(s + 2) % 3][1]);
    }
};

// ------------------------------------------------------------------------------------------------
// LLF flux, rkdg_swe_LLF_flux.hpp:7-60
// ------------------------------------------------------------------------------------------------
void LLF_flux(double gravity, const double qin[3], const double qex[3], double bath, double sp, const double n[2],
              double F[3]) {
    double h_in = qin[0] + bath;
    double u_in = qin[1] / h_in;
    double v_in = qin[2] / h_in;
    double h_ex = qex[0] + bath;
    double u_ex = qex[1] / h_ex;
    double v_ex = qex[2] / h_ex;
    double un_in = u_in * n[0] + v_in * n[1];
    double un_ex = u_ex * n[0] + v_ex * n[1];
    double sp_correction = std::pow(n[0] * sp, 2) + std::pow(n[1], 2);
    double max_eigenvalue = std::max(std::abs(un_in) + std::sqrt(gravity * h_in * sp_correction),
                                     std::abs(un_ex) + std::sqrt(gravity * h_ex * sp_correction));
    double nx = n[0], ny = n[1];
    double uuh_in = u_in * qin[1];
    double vvh_in = v_in * qin[2];
    double uvh_in = u_in * qin[2];
    double pe_in = gravity * (std::pow(qin[0], 2) / 2 + qin[0] * bath);
    double Fin[3], Fex[3];
    Fin[0] = sp * qin[1] * nx + qin[2] * ny;
    Fin[1] = sp * (uuh_in + pe_in) * nx + uvh_in * ny;
    Fin[2] = sp * uvh_in * nx + (vvh_in + pe_in) * ny;
    double uuh_ex = u_ex * qex[1];
    double vvh_ex = v_ex * qex[2];
    double uvh_ex = u_ex * qex[2];
    double pe_ex = gravity * (std::pow(qex[0], 2) / 2 + qex[0] * bath);
    Fex[0] = qex[1] * nx + qex[2] * ny;
    Fex[1] = (uuh_ex + pe_ex) * nx + uvh_ex * ny;
    Fex[2] = uvh_ex * nx + (vvh_ex + pe_ex) * ny;
    for (int i = 0; i < 3; ++i) F[i] = 0.5 * (Fin[i] + Fex[i] + max_eigenvalue * (qin[i] - qex[i]));
}

// land boundary ghost state + LLF, rkdg_swe_bc_land.hpp:68-86
void land_flux(double g, const double n[2], const double qin[3], double bath, double sp, double F[3]) {
    double n_x = n[0], n_y = n[1];
    double t_x = -n_y, t_y = n_x;
    double qn_ex = -(qin[1] * n_x + qin[2] * n_y);
    double qt_ex = qin[1] * t_x + qin[2] * t_y;
    double qex[3];
    qex[0] = qin[0];
    qex[1] = qn_ex * n_x + qt_ex * t_x;
    qex[2] = qn_ex * n_y + qt_ex * t_y;
    LLF_flux(g, qin, qex, bath, sp, n, F);
}

// ------------------------------------------------------------------------------------------------
// Problem state
// ------------------------------------------------------------------------------------------------
struct FaceData {  // SWE::Boundary per element face (swe_data_boundary.hpp)
    vector<double> q_at_gp;  // [var*ngp+gp]
    vector<double> bath, h, sp;
    vector<double> F_hat;  // [var*ngp+gp]
};

struct Elt {
    uint32_t id;
    int node_idx[3];
    uint32_t neighbor_ID[3];
    int neighbor_idx[3];
    uint8_t btype[3];
    Shape shape;
    double detJ, Jinv[2][2];
    vector<double> int_fact, int_phi, int_dphi[2], dphi[2], minv;
    vector<double> gpx, gpy;  // gp global coords
    vector<double> bath;      // modal bathymetry (state[0].aux)
    vector<double> bath_gp, sp_gp, db_gp[2];
    vector<vector<double>> q, rhs, sol;  // per stage [var*nd+dof]
    FaceData face[3];
    // wet/dry (swe_data_wet_dry.hpp)
    bool wet = true;
    double wd_bath_vrtx[3], wd_bath_min;
    // slope limiter (swe_data_slope_limit.hpp)
    double sl_bath_baryctr, sl_bath_vrtx[3];
    double sl_baryctr_coord[2], sl_midpts_coord[3][2], sl_baryctr_neigh_coord[3][2];
    double sl_median[3][2], sl_alpha[3][2], sl_r_sq[3], sl_lengths[3], sl_radius;
    double sl_q_lin[3][3], sl_q_baryctr[3], sl_q_vrtx[3][3], sl_q_midpts[3][3];
    bool sl_wet_neigh[3] = {false, false, false};
    double sl_q_baryctr_neigh[3][3];
    double sl_I = 0.0, sl_perimeter = 0.0;
    bool sl_troubled = false;
    bool limited = false;
    // bottom friction (swe_data_source.hpp): Manning factor g * mean(n)^2
    bool manning = false;
    double g_manning_n_sq = 0.0;
};

struct Intf {
    int in, ex, bin, bex;
    int ngp;
    vector<double> phi_in, phi_ex;          // [dof*ngp+gp]
    vector<double> ipf_in, ipf_ex;          // [gp*nd+dof]
    vector<double> int_fact_in, int_fact_ex;
    double n_in[2];
    vector<double> gpx_in, gpy_in;
    // ISP::Levee (rkdg_swe_is_levee.hpp:36-62): crest height and discharge coefficients at the gp
    bool levee = false;
    vector<double> H_bar_gp, C_subcrit_gp, C_supercrit_gp;
};

struct Bnd {
    int elt, bid, type;
    int ngp;
    vector<double> phi, ipf, int_fact;
    double n[2];
    vector<double> gpx, gpy;
    // BC::Tide / BC::Flow data (rkdg_swe_bc_tide.hpp:9-71): constituents of the face's first node and
    // amplitude / phase at the Gauss points
    vector<double> frequency, forcing_fact, equilib_arg;
    vector<vector<double>> amplitude_gp, phase_gp;
};

struct Problem {
    orc_config cfg;
    Master master;
    dgsw_rk_table rk;
    int p, nd, ns;
    vector<Elt> elts;                      // ascending ID
    std::map<uint32_t, int> id_to_idx;
    vector<Intf> intfs;
    vector<Bnd> bnds;
    // per element, ordered list of edge contributions: (kind 0 intf / 1 bnd, index, side)
    vector<vector<std::array<int, 3>>> contrib;
    int stage = 0;
    int step = 0;
    double t = 0.0;
    double ramp = 1.0;  // ESSPRKStepper::ramp
    double h_o_threshold = 1.0e-6;
    int nthreads = 1;
    dgsw::Rule2D l2rule;
    vector<double> l2phi;

    double stage_time() const { return t + cfg.dt * rk.drk[stage]; }
};

#define OMP_FOR _Pragma("omp parallel for num_threads(P.nthreads) schedule(static)")

// ------------------------------------------------------------------------------------------------
// Mesh metadata (preprocessor/mesh_metadata.cpp:3-85) and boundary type lookup
// (ADCIRC_reader/adcirc_format.cpp get_ibtype / has_edge)
// ------------------------------------------------------------------------------------------------
// AdcircFormat::has_edge (adcirc_format.cpp:320-336): looks at every occurrence of n0
bool has_edge(const int32_t* b, const int32_t* e, int32_t n0, int32_t n1) {
    const int32_t* it = std::find(b, e, n0);
    if (it != e) {
        if ((it + 1) != e && *(it + 1) == n1) return true;
        if (it != b && *(it - 1) == n1) return true;
        return has_edge(it + 1, e, n0, n1);
    }
    return false;
}

// AdcircFormat::get_ibtype (adcirc_format.cpp:214-259) over the chains in search order; a levee chain
// (type 129) is its front string then its back string, each searched on its own; a face joining the
// two strings at a barrier end is land (is_levee_end, :338-352)
int get_ibtype(const orc_mesh* m, int32_t n0, int32_t n1) {
    for (int s = 0; s < m->n_segments; ++s) {
        const int32_t* b = m->seg_nodes + m->seg_offsets[s];
        const int32_t* e = m->seg_nodes + m->seg_offsets[s + 1];
        if (m->seg_type[s] == BT_LEVEE) {
            const int32_t* mid = b + (e - b) / 2;
            if (has_edge(b, mid, n0, n1) || has_edge(mid, e, n0, n1)) return BT_LEVEE;
        } else if (has_edge(b, e, n0, n1)) {
            return m->seg_type[s];
        }
    }
    const int32_t lo = std::min(n0, n1), hi = std::max(n0, n1);
    for (int s = 0; s < m->n_segments; ++s) {
        if (m->seg_type[s] != BT_LEVEE) continue;
        const int32_t* b = m->seg_nodes + m->seg_offsets[s];
        const int64_t n = (m->seg_offsets[s + 1] - m->seg_offsets[s]) / 2;
        const int32_t *fr = b, *bk = b + n;
        if ((lo == std::min(fr[0], bk[0]) && hi == std::max(fr[0], bk[0])) ||
            (lo == std::min(fr[n - 1], bk[n - 1]) && hi == std::max(fr[n - 1], bk[n - 1])))
            return BT_LAND;
    }
    return -1;
}

// AdcircFormat::get_internal_node_pair (adcirc_format.cpp:261-318): the node pair across the barrier
std::pair<int32_t, int32_t> internal_node_pair(const orc_mesh* m, int32_t n0, int32_t n1) {
    for (int s = 0; s < m->n_segments; ++s) {
        if (m->seg_type[s] != BT_LEVEE) continue;
        const int64_t n = (m->seg_offsets[s + 1] - m->seg_offsets[s]) / 2;
        const int32_t* fr = m->seg_nodes + m->seg_offsets[s];
        const int32_t* bk = fr + n;
        for (int side = 0; side < 2; ++side) {
            const int32_t* a = side == 0 ? fr : bk;
            const int32_t* o = side == 0 ? bk : fr;
            if (a[0] == n0 && a[1] == n1) return {o[1], o[0]};
            for (int64_t k = 1; k < n - 1; ++k)
                if (a[k] == n0) {
                    if (a[k + 1] == n1) return {o[k + 1], o[k]};
                    if (a[k - 1] == n1) return {o[k - 1], o[k]};
                }
            if (a[n - 1] == n0 && a[n - 2] == n1) return {o[n - 2], o[n - 1]};
        }
    }
    throw std::runtime_error("Fatal Error: back nodes not found to given node_pair");
}

// Tide / flow data of one boundary face: create_boundaries (swe_pre_create_bound.hpp:33-96) takes the
// first .bcis block of the face's type holding both of its nodes (TideBoundary::get_tide_data,
// swe_inputs.hpp:34-49); the BC::Tide / BC::Flow constructors take the constituents of the face's first
// node and the nodal amplitude / phase (rkdg_swe_bc_tide.hpp:33-52), Initialize interpolates them to the
// Gauss points with GetBoundaryPsi's N1 = (1 - z) / 2, N2 = (1 + z) / 2 (shape_straighttriangle.cpp:215-227).
void attach_forcing(const orc_mesh* m, const Elt& E, const dgsw::Rule1D& gl, Bnd& B) {
    const int32_t nodes[2] = {E.node_idx[(B.bid + 1) % 3], E.node_idx[(B.bid + 2) % 3]};
    for (int32_t b = 0; b < m->n_forcing; ++b) {
        const orc_forcing_block& F = m->forcing[b];
        if (F.type != B.type) continue;
        int pos[2] = {-1, -1};
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < F.n_nodes; ++j)
                if (F.nodes[j] == nodes[k]) {
                    if (pos[k] >= 0) throw std::runtime_error("forcing block lists a node twice");
                    pos[k] = j;
                }
        if (pos[0] < 0 || pos[1] < 0) continue;
        const int ncon = F.n_constituents, ngb = (int)gl.z.size();
        B.frequency.assign(F.frequency, F.frequency + ncon);
        B.forcing_fact.assign(F.forcing_fact, F.forcing_fact + ncon);
        B.equilib_arg.assign(F.equilib_arg, F.equilib_arg + ncon);
        B.amplitude_gp.assign(ncon, vector<double>(ngb, 0.0));
        B.phase_gp.assign(ncon, vector<double>(ngb, 0.0));
        for (int con = 0; con < ncon; ++con) {
            const double a[2] = {F.amplitude[(size_t)con * F.n_nodes + pos[0]], F.amplitude[(size_t)con * F.n_nodes + pos[1]]};
            const double ph[2] = {F.phase[(size_t)con * F.n_nodes + pos[0]], F.phase[(size_t)con * F.n_nodes + pos[1]]};
            for (int gp = 0; gp < ngb; ++gp) {
                const double psi[2] = {(1 - gl.z[gp]) / 2, (1 + gl.z[gp]) / 2};
                double sa = 0, sp = 0;
                for (int n = 0; n < 2; ++n) {
                    sa += a[n] * psi[n];
                    sp += ph[n] * psi[n];
                }
                B.amplitude_gp[con][gp] = sa;
                B.phase_gp[con][gp] = sp;
            }
        }
        return;
    }
    throw std::runtime_error(B.type == BT_TIDE ? "Fatal Error: unable to find tide data!\n"
                                               : "Fatal Error: unable to find flow data!\n");
}

// Utilities::almost_equal(a, 0) (utilities/almost_equal.hpp:16-22) with its default factor 100
bool almost_zero(double a) { return std::abs(a) < DBL_EPS * 100; }

int build(Problem& P, const orc_config* cfg, const orc_mesh* m) {
    P.cfg = *cfg;
    P.p = cfg->p;
    if (P.p < 1 || P.p > 4) throw std::runtime_error("unsupported polynomial order");
    P.master.init(P.p);
    P.nd = P.master.nd;
    if (dgsw_rk_table_init(cfg->rk_nstages, cfg->rk_order, &P.rk) != 0)
        throw std::runtime_error("Fatal Error: invalid Runge-Kutta method entered!");
    P.ns = cfg->rk_nstages;
    P.nthreads = cfg->n_threads > 0 ? cfg->n_threads : 1;
    // ESSPRKStepper ctor (explicit_ssp_rk_stepper.cpp:12): ramp 1 if ramp_duration is almost zero, else 0
    P.ramp = almost_zero(cfg->ramp_duration) ? 1.0 : 0.0;
    if (cfg->bottom_friction < 0 || cfg->bottom_friction > 2) throw std::runtime_error("unknown bottom friction type");
    if (cfg->bottom_friction != 0 && cfg->friction_cf < 0.)
        throw std::runtime_error("Fatal Error: Chezy friction coefficient must be postive!");
    if (cfg->bottom_friction == 2 && !m->node_manning_n) throw std::runtime_error("Manning friction needs node n");
    if (cfg->wetting_drying) P.h_o_threshold = 1.0e6 * cfg->h_o * DBL_EPS;  // swe_pre_init_prob_params.hpp:36
    const int ne = (int)m->n_elems;
    // elements in ascending ID order (element storage is an ordered map keyed by ID)
    vector<std::pair<uint32_t, int>> order(ne);
    for (int i = 0; i < ne; ++i) order[i] = {m->elem_ids ? m->elem_ids[i] : (uint32_t)i, i};
    std::sort(order.begin(), order.end());
    P.elts.resize(ne);
    vector<int> src_of(ne);
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        int i = order[k].second;
        src_of[k] = i;
        E.id = order[k].first;
        if (P.id_to_idx.count(E.id)) throw std::runtime_error("duplicate element ID");
        P.id_to_idx[E.id] = k;
        for (int v = 0; v < 3; ++v) {
            E.node_idx[v] = m->elem_nodes[3 * i + v];
            if (E.node_idx[v] < 0 || E.node_idx[v] >= m->n_nodes) throw std::runtime_error("node index out of range");
            for (int c = 0; c < 3; ++c) E.shape.X[v][c] = m->node_xyz[3 * E.node_idx[v] + c];
        }
        // CCW fix-up swaps coordinates, not node IDs (shape_straighttriangle.cpp:4-12)
        if (E.shape.detJ() < 0) std::swap(E.shape.X[0], E.shape.X[2]);
    }
    // edge dictionary: key = min<<32 | max over node IDs of face k (nodes k+1, k+2)
    std::unordered_map<uint64_t, std::pair<std::pair<uint32_t, int>, std::pair<uint32_t, int>>> dict;
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        for (int f = 0; f < 3; ++f) {
            uint32_t a = E.node_idx[(f + 1) % 3], b = E.node_idx[(f + 2) % 3];
            uint64_t key = (uint64_t)std::min(a, b) << 32 | std::max(a, b);
            auto it = dict.find(key);
            if (it != dict.end())
                it->second.second = {E.id, f};
            else
                dict.insert({key, {{E.id, f}, {DEFAULT_ID, 0}}});
        }
    }
    for (auto& kv : dict) {
        auto A = kv.second.first, B = kv.second.second;
        if (B.first != DEFAULT_ID) {
            Elt& EA = P.elts[P.id_to_idx[A.first]];
            Elt& EB = P.elts[P.id_to_idx[B.first]];
            EA.neighbor_ID[A.second] = B.first;
            EA.btype[A.second] = BT_INTERNAL;
            EB.neighbor_ID[B.second] = A.first;
            EB.btype[B.second] = BT_INTERNAL;
        } else {
            Elt& E = P.elts[P.id_to_idx[A.first]];
            int f = A.second;
            int32_t n0 = E.node_idx[(f + 1) % 3], n1 = E.node_idx[(f + 2) % 3];
            int bt = get_ibtype(m, n0, n1);
            if (bt < 0)
                throw std::runtime_error("Fatal Error: boundary not found, unable to assign BOUNDARY_TYPE to given node_pair");
            E.neighbor_ID[f] = DEFAULT_ID;
            E.btype[f] = (uint8_t)bt;
            // the element across an internal barrier (mesh_metadata.cpp:75-82)
            if (bt == BT_LEVEE) {
                auto np = internal_node_pair(m, n0, n1);
                uint64_t key = (uint64_t)(uint32_t)std::min(np.first, np.second) << 32 |
                               (uint32_t)std::max(np.first, np.second);
                auto it = dict.find(key);
                if (it == dict.end()) throw std::runtime_error("Fatal Error: no element across the barrier");
                E.neighbor_ID[f] = it->second.first.first;
            }
        }
    }
    for (auto& E : P.elts)
        for (int f = 0; f < 3; ++f)
            E.neighbor_idx[f] = (E.neighbor_ID[f] == DEFAULT_ID) ? -1 : P.id_to_idx[E.neighbor_ID[f]];

    const Master& M = P.master;
    const int nd = P.nd, ngp = M.ngp;
    // Element::Initialize, element.hpp:167-272
    for (auto& E : P.elts) {
        E.detJ = E.shape.detJ();
        E.shape.Jinv(E.Jinv);
        double aJ = std::abs(E.detJ);
        E.gpx.resize(ngp);
        E.gpy.resize(ngp);
        for (int gp = 0; gp < ngp; ++gp) E.shape.local_to_global(M.rule.z1[gp], M.rule.z2[gp], E.gpx[gp], E.gpy[gp]);
        for (int dir = 0; dir < 2; ++dir) {
            E.dphi[dir].assign(nd * ngp, 0.0);
            for (int gp = 0; gp < ngp; ++gp)
                for (int dof = 0; dof < nd; ++dof) {
                    double d = 0.0;
                    for (int z = 0; z < 2; ++z) d += M.dphi[z][dof * ngp + gp] * E.Jinv[z][dir];
                    E.dphi[dir][dof * ngp + gp] = d;
                }
        }
        E.int_fact.resize(ngp);
        for (int gp = 0; gp < ngp; ++gp) E.int_fact[gp] = M.rule.w[gp] * aJ;
        E.int_phi.resize(ngp * nd);
        for (int i = 0; i < ngp * nd; ++i) E.int_phi[i] = M.int_phi[i] * aJ;
        for (int dir = 0; dir < 2; ++dir) {
            E.int_dphi[dir].assign(ngp * nd, 0.0);
            for (int dof = 0; dof < nd; ++dof)
                for (int gp = 0; gp < ngp; ++gp) {
                    double d = 0;
                    for (int z = 0; z < 2; ++z) d += M.int_dphi[z][gp * nd + dof] * E.Jinv[z][dir];
                    d *= aJ;
                    E.int_dphi[dir][gp * nd + dof] = d;
                }
        }
        E.minv.resize(nd);
        for (int dof = 0; dof < nd; ++dof) E.minv[dof] = M.minv[dof] / aJ;
        E.q.assign(P.ns + 1, vector<double>(3 * nd, 0.0));
        E.rhs.assign(P.ns + 1, vector<double>(3 * nd, 0.0));
        E.sol.assign(P.ns + 1, vector<double>(3 * nd, 0.0));
    }

    // raw boundaries and interface/boundary creation (swe_pre_create_intface.hpp, swe_pre_create_bound.hpp)
    std::map<std::pair<uint32_t, uint32_t>, std::pair<int, int>> raw_internal;  // (id, neigh id) -> (elt, face)
    std::map<std::pair<uint32_t, uint32_t>, std::pair<int, int>> raw_levee;
    std::map<int, std::map<std::pair<uint32_t, uint32_t>, std::pair<int, int>>> raw_bound;
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        for (int f = 0; f < 3; ++f) {
            if (E.btype[f] == BT_INTERNAL)
                raw_internal.emplace(std::make_pair(E.id, E.neighbor_ID[f]), std::make_pair(k, f));
            else if (E.btype[f] == BT_LEVEE)
                raw_levee.emplace(std::make_pair(E.id, E.neighbor_ID[f]), std::make_pair(k, f));
            else
                raw_bound[E.btype[f]].emplace(std::make_pair(E.id, (uint32_t)f), std::make_pair(k, f));
        }
    }
    const dgsw::Rule1D gl = dgsw::gauss_legendre_degree(2 * P.p + 1);
    const int ngb = (int)gl.w.size();
    auto make_face_data = [&](Elt& E, int f) {
        FaceData& F = E.face[f];
        F.q_at_gp.assign(3 * ngb, 0.0);
        F.bath.assign(ngb, 0.0);
        F.h.assign(ngb, 0.0);
        F.sp.assign(ngb, 1.0);
        F.F_hat.assign(3 * ngb, 0.0);
    };
    for (auto& E : P.elts)
        for (int f = 0; f < 3; ++f) make_face_data(E, f);
    // levee_is_data keyed (front, back); swe_pre_create_intface.hpp:50-66 looks a face's node pair up in
    // both orders
    std::map<std::pair<int32_t, int32_t>, int32_t> levee_data;
    for (int32_t k = 0; k < m->n_levee_pairs; ++k) levee_data[{m->levee_nodes[2 * k], m->levee_nodes[2 * k + 1]}] = k;
    auto create_interfaces = [&](std::map<std::pair<uint32_t, uint32_t>, std::pair<int, int>>& raw, bool levee) {
        auto it = raw.begin();
        while (it != raw.end()) {
            auto key_ex = std::make_pair(it->first.second, it->first.first);
            auto jt = raw.find(key_ex);
            if (jt != raw.end()) {
                Intf I;
                I.in = it->second.first;
                I.bin = it->second.second;
                I.ex = jt->second.first;
                I.bex = jt->second.second;
                I.ngp = ngb;
                const Elt& Ein = P.elts[I.in];
                vector<double> z1i(ngb), z2i(ngb), z1e(ngb), z2e(ngb);
                for (int gp = 0; gp < ngb; ++gp) {
                    bound_to_master(I.bin, gl.z[gp], z1i[gp], z2i[gp]);
                    bound_to_master(I.bex, gl.z[gp], z1e[gp], z2e[gp]);
                }
                I.gpx_in.resize(ngb);
                I.gpy_in.resize(ngb);
                for (int gp = 0; gp < ngb; ++gp) Ein.shape.local_to_global(z1i[gp], z2i[gp], I.gpx_in[gp], I.gpy_in[gp]);
                I.phi_in = get_phi(P.p, z1i, z2i);
                I.phi_ex = get_phi(P.p, z1e, z2e);
                double sJ = Ein.shape.surface_J(I.bin);
                I.int_fact_in.resize(ngb);
                I.int_fact_ex.resize(ngb);
                for (int gp = 0; gp < ngb; ++gp) I.int_fact_in[gp] = I.int_fact_ex[gp] = gl.w[gp] * sJ;
                I.ipf_in.resize(ngb * nd);
                I.ipf_ex.resize(ngb * nd);
                for (int dof = 0; dof < nd; ++dof)
                    for (int gp = 0; gp < ngb; ++gp) {
                        I.ipf_in[gp * nd + dof] = I.phi_in[dof * ngb + gp] * (gl.w[gp] * sJ);
                        I.ipf_ex[gp * nd + dof] = I.phi_ex[dof * ngb + gp] * (gl.w[gp] * sJ);
                    }
                Ein.shape.normal(I.bin, I.n_in);
                if (levee) {
                    const Elt& Eex = P.elts[I.ex];
                    const int32_t ni[2] = {Ein.node_idx[(I.bin + 1) % 3], Ein.node_idx[(I.bin + 2) % 3]};
                    const int32_t nx[2] = {Eex.node_idx[(I.bex + 1) % 3], Eex.node_idx[(I.bex + 2) % 3]};
                    double H[2], Cs[2], Cp[2];
                    for (int node = 0; node < 2; ++node) {
                        auto d = levee_data.find({ni[node], nx[1 - node]});
                        if (d == levee_data.end()) d = levee_data.find({nx[1 - node], ni[node]});
                        if (d == levee_data.end()) throw std::runtime_error("Fatal Error: unable to find levee data!\n");
                        H[node] = m->levee_data[3 * d->second];
                        Cs[node] = m->levee_data[3 * d->second + 1];
                        Cp[node] = m->levee_data[3 * d->second + 2];
                    }
                    I.levee = true;
                    I.H_bar_gp.resize(ngb);
                    I.C_subcrit_gp.resize(ngb);
                    I.C_supercrit_gp.resize(ngb);
                    for (int gp = 0; gp < ngb; ++gp) {  // ComputeBoundaryNodalUgpIN
                        const double psi[2] = {(1 - gl.z[gp]) / 2, (1 + gl.z[gp]) / 2};
                        I.H_bar_gp[gp] = H[0] * psi[0] + H[1] * psi[1];
                        I.C_subcrit_gp[gp] = Cs[0] * psi[0] + Cs[1] * psi[1];
                        I.C_supercrit_gp[gp] = Cp[0] * psi[0] + Cp[1] * psi[1];
                    }
                }
                P.intfs.push_back(std::move(I));
            }
            it = raw.erase(it);
        }
    };
    // internal interfaces, then levee interfaces (swe_pre_create_intface.hpp:13-82)
    create_interfaces(raw_internal, false);
    create_interfaces(raw_levee, true);
    // boundaries grouped by condition type in the order Land, Tide, Flow, Function
    // (ProblemBoundaryTypes tuple order, rkdg_swe_problem.hpp:46); outflow faces get no boundary object
    for (int bt : {BT_LAND, BT_TIDE, BT_FLOW, BT_FUNCTION}) {
        auto it = raw_bound.find(bt);
        if (it == raw_bound.end()) continue;
        for (auto& kv : it->second) {
            Bnd B;
            B.elt = kv.second.first;
            B.bid = kv.second.second;
            B.type = bt;
            B.ngp = ngb;
            const Elt& E = P.elts[B.elt];
            vector<double> z1(ngb), z2(ngb);
            for (int gp = 0; gp < ngb; ++gp) bound_to_master(B.bid, gl.z[gp], z1[gp], z2[gp]);
            B.gpx.resize(ngb);
            B.gpy.resize(ngb);
            for (int gp = 0; gp < ngb; ++gp) E.shape.local_to_global(z1[gp], z2[gp], B.gpx[gp], B.gpy[gp]);
            B.phi = get_phi(P.p, z1, z2);
            double sJ = E.shape.surface_J(B.bid);
            B.int_fact.resize(ngb);
            for (int gp = 0; gp < ngb; ++gp) B.int_fact[gp] = gl.w[gp] * sJ;
            B.ipf.resize(ngb * nd);
            for (int dof = 0; dof < nd; ++dof)
                for (int gp = 0; gp < ngb; ++gp) B.ipf[gp * nd + dof] = B.phi[dof * ngb + gp] * (gl.w[gp] * sJ);
            E.shape.normal(B.bid, B.n);
            if (bt == BT_TIDE || bt == BT_FLOW) attach_forcing(m, E, gl, B);
            P.bnds.push_back(std::move(B));
        }
    }
    for (auto& kv : raw_bound)
        if (kv.first != BT_LAND && kv.first != BT_FUNCTION && kv.first != BT_OUTFLOW)
            if (kv.first != BT_TIDE && kv.first != BT_FLOW)
                throw std::runtime_error("unsupported boundary type");

    // per-element contribution order: interfaces in creation order, then boundaries
    P.contrib.assign(ne, {});
    for (int i = 0; i < (int)P.intfs.size(); ++i) {
        P.contrib[P.intfs[i].in].push_back({0, i, 0});
        P.contrib[P.intfs[i].ex].push_back({0, i, 1});
    }
    for (int i = 0; i < (int)P.bnds.size(); ++i) P.contrib[P.bnds[i].elt].push_back({1, i, 0});

    // ---------------- initialize_data_serial, swe_pre_init_data.hpp:9-327 ----------------
    const double cos_phi_o = std::cos(cfg->sp_lat0_deg * REF_PI / 180.0);  // swe_pre_init_data.hpp:40
    auto sp_of = [&](double y) { return cfg->spherical ? cos_phi_o / std::cos(y / cfg->sp_R) : 1.0; };
    vector<double> psi_gp(3 * ngp);  // shape.psi_gp (node x gp)
    for (int gp = 0; gp < ngp; ++gp) {
        double ps[3];
        Shape::psi(M.rule.z1[gp], M.rule.z2[gp], ps);
        for (int n = 0; n < 3; ++n) psi_gp[n * ngp + gp] = ps[n];
    }
    // L2ProjectionNode: ((nodal * psi_gp) * int_phi_fact) * m_inv
    auto l2proj_node = [&](const Elt& E, const double nodal[3], double* out) {
        vector<double> a(ngp, 0.0), b(nd, 0.0);
        for (int gp = 0; gp < ngp; ++gp) {
            double s = 0;
            for (int n = 0; n < 3; ++n) s += nodal[n] * psi_gp[n * ngp + gp];
            a[gp] = s;
        }
        for (int dof = 0; dof < nd; ++dof) {
            double s = 0;
            for (int gp = 0; gp < ngp; ++gp) s += a[gp] * E.int_phi[gp * nd + dof];
            b[dof] = s;
        }
        for (int dof = 0; dof < nd; ++dof) out[dof] = b[dof] * E.minv[dof];
    };
    OMP_FOR
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        double z[3] = {E.shape.X[0][2], E.shape.X[1][2], E.shape.X[2][2]};
        E.bath.assign(nd, 0.0);
        l2proj_node(E, z, E.bath.data());
        E.bath_gp.assign(ngp, 0.0);
        E.sp_gp.assign(ngp, 1.0);
        for (int d = 0; d < 2; ++d) E.db_gp[d].assign(ngp, 0.0);
        for (int gp = 0; gp < ngp; ++gp) {
            double s = 0, sx = 0, sy = 0;
            for (int dof = 0; dof < nd; ++dof) {
                s += E.bath[dof] * M.phi[dof * ngp + gp];
                sx += E.bath[dof] * E.dphi[0][dof * ngp + gp];
                sy += E.bath[dof] * E.dphi[1][dof * ngp + gp];
            }
            E.bath_gp[gp] = s;
            E.db_gp[0][gp] = sx;
            E.db_gp[1][gp] = sy;
            double y = 0;
            for (int n = 0; n < 3; ++n) y += E.shape.X[n][1] * psi_gp[n * ngp + gp];
            E.sp_gp[gp] = sp_of(y);
        }
        double* q0 = E.q[0].data();
        if (cfg->ic_type == 0) {
            for (int v = 0; v < 3; ++v) {
                double nodal[3] = {cfg->ic_const[v], cfg->ic_const[v], cfg->ic_const[v]};
                l2proj_node(E, nodal, q0 + v * nd);
            }
        } else {
            // L2ProjectionF: (f_gp * int_phi_fact) * m_inv
            vector<double> fg(3 * ngp);
            for (int gp = 0; gp < ngp; ++gp) {
                dgsw_fn3 f = dgsw_fn_ic(cfg->function_set, cfg->fn_params, 0.0, E.gpx[gp], E.gpy[gp]);
                fg[0 * ngp + gp] = f.ze;
                fg[1 * ngp + gp] = f.qx;
                fg[2 * ngp + gp] = f.qy;
            }
            for (int v = 0; v < 3; ++v)
                for (int dof = 0; dof < nd; ++dof) {
                    double s = 0;
                    for (int gp = 0; gp < ngp; ++gp) s += fg[v * ngp + gp] * E.int_phi[gp * nd + dof];
                    q0[v * nd + dof] = s * E.minv[dof];
                }
        }
    }
    // edge bathymetry and sp (swe_pre_init_data.hpp:67-131)
    for (auto& I : P.intfs) {
        Elt& Ei = P.elts[I.in];
        Elt& Ee = P.elts[I.ex];
        FaceData& Fi = Ei.face[I.bin];
        FaceData& Fe = Ee.face[I.bex];
        for (int gp = 0; gp < ngb; ++gp) {
            double si = 0, se = 0;
            for (int dof = 0; dof < nd; ++dof) {
                si += Ei.bath[dof] * I.phi_in[dof * ngb + gp];
                se += Ee.bath[dof] * I.phi_ex[dof * ngb + gp];
            }
            Fi.bath[gp] = si;
            Fe.bath[gp] = se;
        }
        for (int gp = 0; gp < ngb; ++gp) {
            int gpe = ngb - gp - 1;
            double y = 0;
            if (cfg->spherical) {
                double z1, z2, ps[3];
                bound_to_master(I.bin, gl.z[gp], z1, z2);
                Shape::psi(z1, z2, ps);
                for (int n = 0; n < 3; ++n) y += Ei.shape.X[n][1] * ps[n];
            }
            Fi.sp[gp] = sp_of(y);
            Fe.sp[gpe] = sp_of(y);
        }
    }
    for (auto& B : P.bnds) {
        Elt& E = P.elts[B.elt];
        FaceData& F = E.face[B.bid];
        for (int gp = 0; gp < ngb; ++gp) {
            double s = 0;
            for (int dof = 0; dof < nd; ++dof) s += E.bath[dof] * B.phi[dof * ngb + gp];
            F.bath[gp] = s;
            double y = 0;
            if (cfg->spherical) {
                double z1, z2, ps[3];
                bound_to_master(B.bid, gl.z[gp], z1, z2);
                Shape::psi(z1, z2, ps);
                for (int n = 0; n < 3; ++n) y += E.shape.X[n][1] * ps[n];
            }
            F.sp[gp] = sp_of(y);
        }
    }
    // wetting-drying initialisation (swe_pre_init_data.hpp:213-250)
    if (cfg->wetting_drying) {
        for (auto& E : P.elts) {
            for (int v = 0; v < 3; ++v) E.wd_bath_vrtx[v] = E.shape.X[v][2];
            E.wd_bath_min = *std::min_element(E.wd_bath_vrtx, E.wd_bath_vrtx + 3);
            double ql[3][3];
            M.basis_to_linear(E.q[0].data(), ql);
            double h[3];
            for (int v = 0; v < 3; ++v) h[v] = ql[0][v] + E.wd_bath_vrtx[v];
            bool set_wet = true;
            for (int v = 0; v < 3; ++v)
                if (h[v] <= cfg->h_o + P.h_o_threshold) {
                    ql[0][v] = cfg->h_o - E.wd_bath_vrtx[v];
                    set_wet = false;
                }
            if (set_wet) {
                E.wet = true;
            } else {
                E.wet = false;
                for (int v = 0; v < 3; ++v) {
                    ql[1][v] = 0.0;
                    ql[2][v] = 0.0;
                }
                for (int var = 0; var < 3; ++var) M.linear_to_basis_row(ql[var], E.q[0].data() + var * nd);
            }
        }
    }
    // slope-limiter geometry (swe_pre_init_data.hpp:252-326)
    if (cfg->slope_limiting) {
        for (auto& E : P.elts) {
            double bl[3] = {E.shape.X[0][2], E.shape.X[1][2], E.shape.X[2][2]};
            double s = 0;
            for (int v = 0; v < 3; ++v) s += bl[v] * M.chi_baryctr[v];
            E.sl_bath_baryctr = s;
            for (int v = 0; v < 3; ++v) E.sl_bath_vrtx[v] = bl[v];
            for (int c = 0; c < 2; ++c)
                E.sl_baryctr_coord[c] = (E.shape.X[0][c] + E.shape.X[1][c] + E.shape.X[2][c]) / 3.0;
            for (int mpt = 0; mpt < 3; ++mpt)
                for (int c = 0; c < 2; ++c)
                    E.sl_midpts_coord[mpt][c] = (E.shape.X[(mpt + 1) % 3][c] + E.shape.X[(mpt + 2) % 3][c]) / 2.0;
            for (int sd = 0; sd < 3; ++sd) E.sl_lengths[sd] = E.shape.length(sd);
            E.sl_radius = E.shape.radius();
            for (int b = 0; b < 3; ++b) {
                double mx = E.sl_midpts_coord[b][0] - E.sl_baryctr_coord[0];
                double my = E.sl_midpts_coord[b][1] - E.sl_baryctr_coord[1];
                double nrm = std::sqrt(mx * mx + my * my);
                E.sl_median[b][0] = mx / nrm;
                E.sl_median[b][1] = my / nrm;
            }
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 2; ++c) E.sl_baryctr_neigh_coord[b][c] = 0.0;
        }
        for (auto& I : P.intfs) {
            Elt& Ei = P.elts[I.in];
            Elt& Ee = P.elts[I.ex];
            for (int c = 0; c < 2; ++c) {
                Ei.sl_baryctr_neigh_coord[I.bin][c] = Ee.sl_baryctr_coord[c];
                Ee.sl_baryctr_neigh_coord[I.bex][c] = Ei.sl_baryctr_coord[c];
            }
        }
        for (auto& B : P.bnds) {
            Elt& E = P.elts[B.elt];
            for (int c = 0; c < 2; ++c)
                E.sl_baryctr_neigh_coord[B.bid][c] = 2.0 * E.sl_midpts_coord[B.bid][c] - E.sl_baryctr_coord[c];
        }
        for (auto& E : P.elts) {
            for (int b = 0; b < 3; ++b) {
                int e1 = b, e2 = (b + 1) % 3;
                double A[2][2];
                A[0][0] = E.sl_baryctr_neigh_coord[e1][0] - E.sl_baryctr_coord[0];
                A[1][0] = E.sl_baryctr_neigh_coord[e1][1] - E.sl_baryctr_coord[1];
                A[0][1] = E.sl_baryctr_neigh_coord[e2][0] - E.sl_baryctr_coord[0];
                A[1][1] = E.sl_baryctr_neigh_coord[e2][1] - E.sl_baryctr_coord[1];
                double bb[2] = {E.sl_midpts_coord[b][0] - E.sl_baryctr_coord[0],
                                E.sl_midpts_coord[b][1] - E.sl_baryctr_coord[1]};
                double invdet = 1.0 / (A[0][0] * A[1][1] - A[1][0] * A[0][1]);
                double Ai[2][2] = {{A[1][1] * invdet, -A[0][1] * invdet}, {-A[1][0] * invdet, A[0][0] * invdet}};
                E.sl_alpha[b][0] = Ai[0][0] * bb[0] + Ai[0][1] * bb[1];
                E.sl_alpha[b][1] = Ai[1][0] * bb[0] + Ai[1][1] * bb[1];
                E.sl_r_sq[b] = bb[0] * bb[0] + bb[1] * bb[1];
            }
        }
    }
    // Manning n per element (swe_pre_init_data.hpp:165-196): g * (mean of the three nodal n)^2
    if (cfg->bottom_friction == 2)
        for (auto& E : P.elts) {
            double n[3];
            for (int v = 0; v < 3; ++v) n[v] = m->node_manning_n[E.node_idx[v]];
            E.manning = true;
            E.g_manning_n_sq = cfg->g * std::pow(std::accumulate(n, n + 3, 0.0) / 3, 2);
        }
    // L2-error rule (Element::ComputeResidualL2 asks for degree 20)
    P.l2rule = dgsw::triangle_rule(20);
    P.l2phi = get_phi(P.p, P.l2rule.z1, P.l2rule.z2);
    (void)src_of;
    return 0;
}

// ------------------------------------------------------------------------------------------------
// stage kernels
// ------------------------------------------------------------------------------------------------
void volume_source(Problem& P, Elt& E) {  // rkdg_swe_proc_volume.hpp:9-35, rkdg_swe_proc_source.hpp:9-18
    const Master& M = P.master;
    const int nd = P.nd, ngp = M.ngp, st = P.stage;
    const double g = P.cfg.g;
    double* rhs = E.rhs[st].data();
    const double* q = E.q[st].data();
    std::fill(rhs, rhs + 3 * nd, 0.0);
    if (!E.wet) return;
    double qg[3][32], Fx[3][32], Fy[3][32];
    for (int v = 0; v < 3; ++v)
        for (int gp = 0; gp < ngp; ++gp) {
            double s = 0;
            for (int dof = 0; dof < nd; ++dof) s += q[v * nd + dof] * M.phi[dof * ngp + gp];
            qg[v][gp] = s;
        }
    for (int gp = 0; gp < ngp; ++gp) {  // swe_flux.hpp:5-25
        double h = qg[0][gp] + E.bath_gp[gp];
        double u = qg[1][gp] / h, vv = qg[2][gp] / h;
        double uuh = u * qg[1][gp], vvh = vv * qg[2][gp], uvh = u * qg[2][gp];
        double pe = g * (0.5 * qg[0][gp] * qg[0][gp] + qg[0][gp] * E.bath_gp[gp]);
        Fx[0][gp] = qg[1][gp];
        Fx[1][gp] = uuh + pe;
        Fx[2][gp] = uvh;
        Fy[0][gp] = qg[2][gp];
        Fy[1][gp] = uvh;
        Fy[2][gp] = vvh + pe;
        for (int v = 0; v < 3; ++v) Fx[v][gp] = E.sp_gp[gp] * Fx[v][gp];
    }
    for (int v = 0; v < 3; ++v)
        for (int dof = 0; dof < nd; ++dof) {
            double sx = 0, sy = 0;
            for (int gp = 0; gp < ngp; ++gp) sx += Fx[v][gp] * E.int_dphi[0][gp * nd + dof];
            for (int gp = 0; gp < ngp; ++gp) sy += Fy[v][gp] * E.int_dphi[1][gp * nd + dof];
            rhs[v * nd + dof] = sx + sy;
        }
    // source (swe_source.hpp:9-27)
    double S[3][32];
    double t = P.stage_time();
    for (int gp = 0; gp < ngp; ++gp) {
        S[0][gp] = 0.0;
        S[1][gp] = g * (E.db_gp[0][gp] * qg[0][gp]);
        S[2][gp] = g * (E.db_gp[1][gp] * qg[0][gp]);
    }
    if (P.cfg.function_source) {
        for (int gp = 0; gp < ngp; ++gp) {
            dgsw_fn3 f = dgsw_fn_source(P.cfg.function_set, P.cfg.fn_params, t, E.gpx[gp], E.gpy[gp]);
            S[0][gp] += f.ze;
            S[1][gp] += f.qx;
            S[2][gp] += f.qy;
        }
    }
    if (P.cfg.bottom_friction != 0) {  // swe_source.hpp:29-51
        for (int gp = 0; gp < ngp; ++gp) {
            double Cf = P.cfg.friction_cf;
            const double h = qg[0][gp] + E.bath_gp[gp];
            const double u = qg[1][gp] / h, v = qg[2][gp] / h;
            if (E.manning) {
                Cf = E.g_manning_n_sq / std::pow(h, 1.0 / 3.0);
                if (Cf < P.cfg.friction_cf) Cf = P.cfg.friction_cf;
            }
            const double stress = Cf * std::hypot(u, v) / h;
            S[1][gp] -= stress * qg[1][gp];
            S[2][gp] -= stress * qg[2][gp];
        }
    }
    for (int v = 0; v < 3; ++v)
        for (int dof = 0; dof < nd; ++dof) {
            double s = 0;
            for (int gp = 0; gp < ngp; ++gp) s += S[v][gp] * E.int_phi[gp * nd + dof];
            rhs[v * nd + dof] += s;
        }
}

void trace(const double* q, const vector<double>& phi, int nd, int ngb, double* out) {
    for (int v = 0; v < 3; ++v)
        for (int gp = 0; gp < ngb; ++gp) {
            double s = 0;
            for (int dof = 0; dof < nd; ++dof) s += q[v * nd + dof] * phi[dof * ngb + gp];
            out[v * ngb + gp] = s;
        }
}

// interface flux, rkdg_swe_proc_intface.hpp:7-27 + rkdg_swe_is_internal.hpp:26-95
// BC::Land::GetEX (rkdg_swe_bc_land.hpp:88-104)
void land_ex(const double n[2], const double q[3], double qe[3]) {
    const double tx = -n[1], ty = n[0];
    const double qn = -(q[1] * n[0] + q[2] * n[1]);
    const double qt = q[1] * tx + q[2] * ty;
    qe[0] = q[0];
    qe[1] = qn * n[0] + qt * tx;
    qe[2] = qn * n[1] + qt * ty;
}

// ISP::Levee::ComputeFlux (rkdg_swe_is_levee.hpp:64-175)
void levee_flux(Problem& P, Intf& I, FaceData& Bi, FaceData& Be, const double n_in[2], const double n_ex[2],
                bool wet_in, bool wet_ex) {
    const int ngb = I.ngp;
    const double H_tolerance = 0.01, G = P.cfg.g;
    double q_in_ex[3] = {0, 0, 0}, q_ex_ex[3] = {0, 0, 0};
    for (int gp = 0; gp < ngb; ++gp) {
        const int gp_ex = ngb - gp - 1;
        const double H = I.H_bar_gp[gp], Csub = I.C_subcrit_gp[gp], Csup = I.C_supercrit_gp[gp];
        double gravity_in = G, gravity_ex = G;
        double qi[3], qe[3];
        for (int v = 0; v < 3; ++v) {
            qi[v] = Bi.q_at_gp[v * ngb + gp];
            qe[v] = Be.q_at_gp[v * ngb + gp_ex];
        }
        const double h_in = qi[0] - H, h_ex = qe[0] - H;
        if ((h_in <= H_tolerance && h_ex <= H_tolerance) || std::abs(h_in - h_ex) <= H_tolerance) {
            land_ex(n_in, qi, q_in_ex);
            land_ex(n_ex, qe, q_ex_ex);
        } else if (h_in > h_ex) {
            const double nx = n_in[0], ny = n_in[1], tx = -ny, ty = nx;
            double qn, qt;
            if (h_ex > 2.0 * h_in / 3.0) {
                qn = Csub * h_ex * std::sqrt(2.0 * G * (h_in - h_ex));
                qt = 0.0;
            } else {
                qn = Csup * (2.0 * h_in / 3.0) * std::sqrt(G * (2.0 * h_in / 3.0));
                qt = 0.0;
            }
            q_in_ex[0] = qi[0];
            q_in_ex[1] = qn * nx + qt * tx;
            q_in_ex[2] = qn * ny + qt * ty;
            q_ex_ex[0] = qe[0];
            q_ex_ex[1] = q_in_ex[1];
            q_ex_ex[2] = q_in_ex[2];
            if (!wet_ex) gravity_ex = 0.0;
        } else if (h_in < h_ex) {
            const double nx = n_ex[0], ny = n_ex[1], tx = -ny, ty = nx;
            double qn, qt;
            if (h_in > 2.0 * h_ex / 3.0) {
                qn = Csub * h_in * std::sqrt(2.0 * G * (h_ex - h_in));
                qt = 0.0;
            } else {
                qn = Csup * (2.0 * h_ex / 3.0) * std::sqrt(G * (2.0 * h_ex / 3.0));
                qt = 0.0;
            }
            q_ex_ex[0] = qe[0];
            q_ex_ex[1] = qn * nx + qt * tx;
            q_ex_ex[2] = qn * ny + qt * ty;
            q_in_ex[0] = qi[0];
            q_in_ex[1] = q_ex_ex[1];
            q_in_ex[2] = q_ex_ex[2];
            if (!wet_in) gravity_in = 0.0;
        }
        double Fi[3], Fe[3];
        LLF_flux(gravity_in, qi, q_in_ex, Bi.bath[gp], Bi.sp[gp], n_in, Fi);
        LLF_flux(gravity_ex, qe, q_ex_ex, Be.bath[gp_ex], Be.sp[gp_ex], n_ex, Fe);
        for (int v = 0; v < 3; ++v) {
            Bi.F_hat[v * ngb + gp] = Fi[v];
            Be.F_hat[v * ngb + gp_ex] = Fe[v];
        }
    }
}

void interface_flux(Problem& P, Intf& I) {
    Elt& Ei = P.elts[I.in];
    Elt& Ee = P.elts[I.ex];
    const int st = P.stage, nd = P.nd, ngb = I.ngp;
    FaceData& Bi = Ei.face[I.bin];
    FaceData& Be = Ee.face[I.bex];
    if (!(Ei.wet || Ee.wet)) return;
    trace(Ei.q[st].data(), I.phi_in, nd, ngb, Bi.q_at_gp.data());
    trace(Ee.q[st].data(), I.phi_ex, nd, ngb, Be.q_at_gp.data());
    const double g = P.cfg.g;
    const bool wet_in = Ei.wet, wet_ex = Ee.wet;
    const double n_in[2] = {I.n_in[0], I.n_in[1]};
    const double n_ex[2] = {-I.n_in[0], -I.n_in[1]};
    if (I.levee) {
        levee_flux(P, I, Bi, Be, n_in, n_ex, wet_in, wet_ex);
        return;
    }
    for (int gp = 0; gp < ngb; ++gp) {
        int ge = ngb - gp - 1;
        double qi[3], qe[3], Fi[3], Fe[3];
        for (int v = 0; v < 3; ++v) {
            qi[v] = Bi.q_at_gp[v * ngb + gp];
            qe[v] = Be.q_at_gp[v * ngb + ge];
        }
        LLF_flux(g, qi, qe, Bi.bath[gp], Bi.sp[gp], n_in, Fi);
        for (int v = 0; v < 3; ++v) Fe[v] = -Fi[v];
        if (Fi[0] > 1e-12) {
            if (!wet_in) {
                for (int v = 0; v < 3; ++v) Fi[v] = 0.0;
                land_flux(g, n_ex, qe, Be.bath[ge], Be.sp[ge], Fe);
            } else if (!wet_ex) {
                LLF_flux(0.0, qe, qi, Be.bath[ge], Be.sp[ge], n_ex, Fe);
                Fe[0] = -Fi[0];
            }
        } else if (Fi[0] < -1e-12) {
            if (!wet_ex) {
                for (int v = 0; v < 3; ++v) Fe[v] = 0.0;
                land_flux(g, n_in, qi, Bi.bath[gp], Bi.sp[gp], Fi);
            } else if (!wet_in) {
                LLF_flux(0.0, qi, qe, Bi.bath[gp], Bi.sp[gp], n_in, Fi);
                Fi[0] = -Fe[0];
            }
        }
        for (int v = 0; v < 3; ++v) {
            Bi.F_hat[v * ngb + gp] = Fi[v];
            Be.F_hat[v * ngb + ge] = Fe[v];
        }
    }
}

// boundary flux, rkdg_swe_proc_bound.hpp:7-20 + BC::Land (:41-66) / BC::Tide / BC::Flow / BC::Function (:27-60)
void boundary_flux(Problem& P, Bnd& B) {
    Elt& E = P.elts[B.elt];
    if (!E.wet) return;
    const int st = P.stage, nd = P.nd, ngb = B.ngp;
    FaceData& F = E.face[B.bid];
    trace(E.q[st].data(), B.phi, nd, ngb, F.q_at_gp.data());
    const double g = P.cfg.g;
    double t = P.stage_time();
    for (int gp = 0; gp < ngb; ++gp) {
        double qi[3], Fh[3];
        for (int v = 0; v < 3; ++v) qi[v] = F.q_at_gp[v * ngb + gp];
        if (B.type == BT_LAND) {
            land_flux(g, B.n, qi, F.bath[gp], F.sp[gp], Fh);
        } else if (B.type == BT_TIDE || B.type == BT_FLOW) {
            // BC::Tide / BC::Flow ComputeFlux (rkdg_swe_bc_tide.hpp:73-100, rkdg_swe_bc_flow.hpp:72-102)
            double forced = 0.0;
            for (size_t con = 0; con < B.frequency.size(); ++con)
                forced += P.ramp * B.forcing_fact[con] * B.amplitude_gp[con][gp] *
                          cos(B.frequency[con] * t + (B.equilib_arg[con] - B.phase_gp[con][gp]) * REF_PI / 180);
            double qe[3];
            if (B.type == BT_TIDE) {
                qe[0] = forced;
                qe[1] = qi[1];
                qe[2] = qi[2];
            } else {
                qe[0] = qi[0];
                qe[1] = forced * B.n[0];
                qe[2] = forced * B.n[1];
            }
            LLF_flux(g, qi, qe, F.bath[gp], F.sp[gp], B.n, Fh);
        } else {
            dgsw_fn3 f = dgsw_fn_ic(P.cfg.function_set, P.cfg.fn_params, t, B.gpx[gp], B.gpy[gp]);
            double qe[3] = {f.ze, f.qx, f.qy};
            LLF_flux(g, qi, qe, F.bath[gp], F.sp[gp], B.n, Fh);
        }
        for (int v = 0; v < 3; ++v) F.F_hat[v * ngb + gp] = Fh[v];
    }
}

void apply_contributions(Problem& P, int k) {
    Elt& E = P.elts[k];
    const int nd = P.nd, st = P.stage;
    double* rhs = E.rhs[st].data();
    for (auto& c : P.contrib[k]) {
        const vector<double>* ipf;
        const FaceData* F;
        int ngb;
        if (c[0] == 0) {
            const Intf& I = P.intfs[c[1]];
            if (!(P.elts[I.in].wet || P.elts[I.ex].wet)) continue;
            ipf = c[2] == 0 ? &I.ipf_in : &I.ipf_ex;
            F = c[2] == 0 ? &E.face[I.bin] : &E.face[I.bex];
            ngb = I.ngp;
        } else {
            const Bnd& B = P.bnds[c[1]];
            if (!E.wet) continue;
            ipf = &B.ipf;
            F = &E.face[B.bid];
            ngb = B.ngp;
        }
        for (int v = 0; v < 3; ++v)
            for (int dof = 0; dof < nd; ++dof) {
                double s = 0;
                for (int gp = 0; gp < ngb; ++gp) s += F->F_hat[v * ngb + gp] * (*ipf)[gp * nd + dof];
                rhs[v * nd + dof] -= s;
            }
    }
}

// wetting/drying, swe_post_wet_dry.hpp:6-145 (state index = current stage after ++stepper)
void wetting_drying(const Master& M, double h_o, double h_o_threshold, const double bath_vrtx[3], double bath_min,
                    double* q, bool& wet) {
    const int nd = M.nd;
    double qv[3][3];
    M.basis_to_linear(q, qv);
    double h[3];
    int ndry = 0;
    for (int v = 0; v < 3; ++v) {
        h[v] = qv[0][v] + bath_vrtx[v];
        if (h[v] <= h_o + h_o_threshold) ++ndry;
    }
    double h_avg = (0.0 + h[0] + h[1] + h[2]) / 3;
    if (h_avg <= h_o_threshold) h_avg = h_o_threshold;
    bool set_wet = false, set_dry = false, check = false;
    if (ndry == 0) {
        if (wet) return;
        check = true;
    } else if (ndry == 3) {
        for (int v = 0; v < 3; ++v) {
            qv[0][v] = h_avg - bath_vrtx[v];
            qv[1][v] = 0.0;
            qv[2][v] = 0.0;
        }
        wet = false;
        for (int var = 0; var < 3; ++var) M.linear_to_basis_row(qv[var], q + var * nd);
        return;
    } else {
        if (h_avg <= h_o + h_o_threshold) {
            for (int v = 0; v < 3; ++v) {
                qv[0][v] = h_avg - bath_vrtx[v];
                qv[1][v] = 0;
                qv[2][v] = 0;
            }
        } else {
            int hmin = (int)(std::min_element(h, h + 3) - h);
            int hmax = (int)(std::max_element(h, h + 3) - h);
            int hmid = 3 - hmax - hmin;
            double ht[3];
            ht[hmin] = h_o;
            ht[hmid] = std::max(h_o, h[hmid] - (ht[hmin] - h[hmin]) / 2);
            ht[hmax] = h[hmax] - (ht[hmin] - h[hmin]) - (ht[hmid] - h[hmid]);
            for (int v = 0; v < 3; ++v) h[v] = ht[v];
            double dqx = 0, dqy = 0;
            int nd_v = 0;
            for (int v = 0; v < 3; ++v)
                if (h[v] <= h_o + h_o_threshold) {
                    nd_v++;
                    dqx += qv[1][v];
                    dqy += qv[2][v];
                    qv[1][v] = 0.0;
                    qv[2][v] = 0.0;
                }
            for (int v = 0; v < 3; ++v) {
                qv[0][v] = h[v] - bath_vrtx[v];
                if (h[v] > h_o + h_o_threshold) {
                    qv[1][v] += dqx / (3 - nd_v);
                    qv[2][v] += dqy / (3 - nd_v);
                }
            }
        }
        for (int var = 0; var < 3; ++var) M.linear_to_basis_row(qv[var], q + var * nd);
        check = true;
    }
    if (check) {
        int hmax = (int)(std::max_element(h, h + 3) - h);
        double ze_hmax = qv[0][hmax];
        if (ze_hmax > h_o - bath_min)
            set_wet = true;
        else
            set_dry = true;
    }
    if (set_dry) {
        wet = false;
        for (int v = 0; v < 3; ++v) {
            qv[1][v] = 0.0;
            qv[2][v] = 0.0;
        }
        for (int var = 0; var < 3; ++var) M.linear_to_basis_row(qv[var], q + var * nd);
    } else if (set_wet) {
        wet = true;
    }
}

// Cockburn-Shu limiter, swe_CS_sl_serial.hpp:9-23, swe_CS_slope_limiter.hpp:9-189,
// swe_trouble_check.hpp:6-116, swe_jacobian.hpp:462-550
void slope_limiter(Problem& P) {
    const Master& M = P.master;
    const int nd = P.nd, st = P.stage, ne = (int)P.elts.size();
    const double g = P.cfg.g;
    OMP_FOR
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        E.limited = false;
        if (E.wet) {
            M.basis_to_linear(E.q[st].data(), E.sl_q_lin);
            for (int var = 0; var < 3; ++var) {
                double s = 0;
                for (int v = 0; v < 3; ++v) s += E.sl_q_lin[var][v] * M.chi_baryctr[v];
                E.sl_q_baryctr[var] = s;
                for (int v = 0; v < 3; ++v) E.sl_q_vrtx[var][v] = E.sl_q_lin[var][v];
                for (int b = 0; b < 3; ++b) {
                    double m = 0;
                    for (int v = 0; v < 3; ++v) m += E.sl_q_lin[var][v] * M.chi_midpts[v][b];
                    E.sl_q_midpts[var][b] = m;
                }
            }
        }
    }
    for (auto& I : P.intfs) {
        Elt& Ei = P.elts[I.in];
        Elt& Ee = P.elts[I.ex];
        Ei.sl_wet_neigh[I.bin] = Ee.wet;
        Ee.sl_wet_neigh[I.bex] = Ei.wet;
        if (Ei.wet && Ee.wet)
            for (int v = 0; v < 3; ++v) {
                Ei.sl_q_baryctr_neigh[I.bin][v] = Ee.sl_q_baryctr[v];
                Ee.sl_q_baryctr_neigh[I.bex][v] = Ei.sl_q_baryctr[v];
            }
    }
    for (auto& B : P.bnds) {
        Elt& E = P.elts[B.elt];
        E.sl_wet_neigh[B.bid] = E.wet;
        if (E.wet)
            for (int v = 0; v < 3; ++v) E.sl_q_baryctr_neigh[B.bid][v] = E.sl_q_baryctr[v];
    }
    // trouble indicator (computed, not used to gate the limiter)
    for (auto& E : P.elts) {
        E.sl_I = 0.0;
        E.sl_perimeter = 0.0;
        E.sl_troubled = false;
    }
    for (auto& I : P.intfs) {
        Elt& Ei = P.elts[I.in];
        Elt& Ee = P.elts[I.ex];
        if (!(Ei.wet || Ee.wet)) continue;
        const int ngb = I.ngp;
        FaceData& Bi = Ei.face[I.bin];
        FaceData& Be = Ee.face[I.bex];
        trace(Ei.q[st].data(), I.phi_in, nd, ngb, Bi.q_at_gp.data());
        trace(Ee.q[st].data(), I.phi_ex, nd, ngb, Be.q_at_gp.data());
        for (int gp = 0; gp < ngb; ++gp) {
            Bi.h[gp] = Bi.q_at_gp[0 * ngb + gp] + Bi.bath[gp];
            Be.h[gp] = Be.q_at_gp[0 * ngb + gp] + Be.bath[gp];
        }
        // normal "momentum" uses rows GlobalCoord::x (= 0) and GlobalCoord::y (= 1) of q_at_gp
        double qn_in_int = 0, qn_ex_int = 0;
        for (int gp = 0; gp < ngb; ++gp) {
            double qn_in = I.n_in[0] * Bi.q_at_gp[0 * ngb + gp] + I.n_in[1] * Bi.q_at_gp[1 * ngb + gp];
            double qn_ex = -I.n_in[0] * Be.q_at_gp[0 * ngb + gp] + -I.n_in[1] * Be.q_at_gp[1 * ngb + gp];
            qn_in_int += qn_in * I.int_fact_in[gp];
            qn_ex_int += qn_ex * I.int_fact_ex[gp];
        }
        if (qn_in_int < 0.0) {
            double s = 0;
            for (int gp = 0; gp < ngb; ++gp) s += (Bi.h[gp] - Be.h[ngb - gp - 1]) * I.int_fact_in[gp];
            Ei.sl_perimeter += Ei.sl_lengths[I.bin];
            Ei.sl_I += std::abs(s);
        }
        if (qn_ex_int < 0.0) {
            double s = 0;
            for (int gp = 0; gp < ngb; ++gp) s += (Be.h[gp] - Bi.h[ngb - gp - 1]) * I.int_fact_ex[gp];
            Ee.sl_perimeter += Ee.sl_lengths[I.bex];
            Ee.sl_I += std::abs(s);
        }
    }
    std::set<uint32_t> area;
    for (auto& E : P.elts) {
        if (E.wet && E.sl_perimeter != 0.0) {
            double h_norm = 0.0;
            for (int v = 0; v < 3; ++v) h_norm = std::max(h_norm, E.sl_q_vrtx[0][v] + E.sl_bath_vrtx[v]);
            E.sl_I /= (std::pow(E.sl_radius, (P.p + 1.0) / 2.0) * E.sl_perimeter * h_norm);
            if (E.sl_I > 1.0) area.insert(E.id);
        }
    }
    for (int pass = 0; pass < 6; ++pass) {
        std::set<uint32_t> na;
        for (auto& E : P.elts)
            if (area.count(E.id)) {
                E.sl_troubled = true;
                na.insert(E.neighbor_ID, E.neighbor_ID + 3);
            }
        area = na;
    }
    // limiting kernel
    const double Mtvb = P.cfg.sl_M, nu = P.cfg.sl_nu;
    OMP_FOR
    for (int k = 0; k < ne; ++k) {
        Elt& E = P.elts[k];
        if (!(E.wet && E.sl_wet_neigh[0] && E.sl_wet_neigh[1] && E.sl_wet_neigh[2])) continue;
        double* q = E.q[st].data();
        double h = E.sl_q_baryctr[0] + E.sl_bath_baryctr;
        double u = E.sl_q_baryctr[1] / h;
        double v = E.sl_q_baryctr[2] / h;
        double delta[3][3];  // (var, bound)
        for (int b = 0; b < 3; ++b) {
            int e1 = b, e2 = (b + 1) % 3;
            double nx = E.sl_median[b][0], ny = E.sl_median[b][1];
            double c = std::sqrt(g * h);
            double R[3][3] = {{1.0, 0.0, 1.0}, {u - c * nx, -ny, u + c * nx}, {v - c * ny, nx, v + c * ny}};
            double un = u * nx + v * ny;
            double iR[3][3] = {{(c + un) / (2 * c), -nx / (2 * c), -ny / (2 * c)},
                               {u * ny - v * nx, -ny, nx},
                               {(c - un) / (2 * c), nx / (2 * c), ny / (2 * c)}};
            auto mv = [&](const double A[3][3], const double x[3], double y[3]) {
                for (int i = 0; i < 3; ++i) {
                    double s = 0;
                    for (int j = 0; j < 3; ++j) s += A[i][j] * x[j];
                    y[i] = s;
                }
            };
            double mid[3] = {E.sl_q_midpts[0][b], E.sl_q_midpts[1][b], E.sl_q_midpts[2][b]};
            double wm[3], w0[3], w1[3], w2[3];
            mv(iR, mid, wm);
            mv(iR, E.sl_q_baryctr, w0);
            mv(iR, E.sl_q_baryctr_neigh[e1], w1);
            mv(iR, E.sl_q_baryctr_neigh[e2], w2);
            double dch[3];
            for (int var = 0; var < 3; ++var) {
                double wt = wm[var] - w0[var];
                double wd = E.sl_alpha[b][0] * (w1[var] - w0[var]) + E.sl_alpha[b][1] * (w2[var] - w0[var]);
                if (std::abs(wt) <= Mtvb * E.sl_r_sq[b])
                    dch[var] = wt;
                else if (std::signbit(wt) == std::signbit(wd))
                    dch[var] = std::copysign(1.0, wt) * std::min(std::abs(wt), std::abs(nu * wd));
                else
                    dch[var] = 0.0;
            }
            double col[3];
            mv(R, dch, col);
            for (int var = 0; var < 3; ++var) delta[var][b] = col[var];
        }
        for (int var = 0; var < 3; ++var) {
            double dsum = 0.0;
            for (int b = 0; b < 3; ++b) dsum += delta[var][b];
            if (dsum != 0.0) {
                double pos = 0.0, neg = 0.0;
                for (int b = 0; b < 3; ++b) {
                    pos += std::max(0.0, delta[var][b]);
                    neg += std::max(0.0, -delta[var][b]);
                }
                double tp = std::min(1.0, neg / pos);
                double tn = std::min(1.0, pos / neg);
                for (int b = 0; b < 3; ++b)
                    delta[var][b] = tp * std::max(0.0, delta[var][b]) - tn * std::max(0.0, -delta[var][b]);
            }
        }
        const double T[3][3] = {{-1.0, 1.0, 1.0}, {1.0, -1.0, 1.0}, {1.0, 1.0, -1.0}};
        double qv[3][3];
        for (int var = 0; var < 3; ++var)
            for (int vx = 0; vx < 3; ++vx) {
                double s = 0;
                for (int b = 0; b < 3; ++b) s += delta[var][b] * T[b][vx];
                qv[var][vx] = E.sl_q_baryctr[var] + s;
            }
        for (int var = 0; var < 3; ++var) {
            double d2 = 0, n2 = 0;
            for (int vx = 0; vx < 3; ++vx) {
                double d = qv[var][vx] - E.sl_q_lin[var][vx];
                d2 += d * d;
                n2 += E.sl_q_lin[var][vx] * E.sl_q_lin[var][vx];
            }
            if (std::sqrt(d2) / std::sqrt(n2) > 1.0e-12) {
                M.linear_to_basis_row(qv[var], q + var * nd);
                E.limited = true;
            }
        }
    }
}

int do_stage(Problem& P) {
    const int ne = (int)P.elts.size();
    const int nI = (int)P.intfs.size(), nB = (int)P.bnds.size();
    OMP_FOR
    for (int k = 0; k < ne; ++k) volume_source(P, P.elts[k]);
    OMP_FOR
    for (int i = 0; i < nI; ++i) interface_flux(P, P.intfs[i]);
    OMP_FOR
    for (int i = 0; i < nB; ++i) boundary_flux(P, P.bnds[i]);
    const int st = P.stage, nd = P.nd, ns = P.ns;
    const double dt = P.cfg.dt;
    OMP_FOR
    for (int k = 0; k < ne; ++k) {
        apply_contributions(P, k);
        Elt& E = P.elts[k];
        // solution = rhs * m_inv (element.hpp:502-505); UpdateState (explicit_ssp_rk_stepper.hpp:67-80)
        for (int v = 0; v < 3; ++v)
            for (int dof = 0; dof < nd; ++dof) E.sol[st][v * nd + dof] = E.rhs[st][v * nd + dof] * E.minv[dof];
        double* nq = E.q[st + 1].data();
        for (int i = 0; i < 3 * nd; ++i) nq[i] = 0.0;
        for (int s = 0; s <= st; ++s) {
            const double a = P.rk.ark[st][s], bdt = dt * P.rk.brk[st][s];
            for (int i = 0; i < 3 * nd; ++i) nq[i] += a * E.q[s][i] + bdt * E.sol[s][i];
        }
        if (st + 1 == ns) std::swap(E.q[0], E.q[ns]);
    }
    // ++stepper (explicit_ssp_rk_stepper.hpp:49-65)
    P.stage = (P.stage + 1) % P.ns;
    if (P.stage == 0) {
        P.t += dt;
        P.step++;
    }
    if (!almost_zero(P.cfg.ramp_duration)) P.ramp = std::tanh(2 * (P.stage_time() / 86400) / P.cfg.ramp_duration);
    if (P.cfg.wetting_drying) {
        OMP_FOR
        for (int k = 0; k < ne; ++k) {
            Elt& E = P.elts[k];
            wetting_drying(P.master, P.cfg.h_o, P.h_o_threshold, E.wd_bath_vrtx, E.wd_bath_min, E.q[P.stage].data(),
                           E.wet);
        }
    }
    if (P.cfg.slope_limiting) slope_limiter(P);
    // scrutinize_solution (swe_post_scrutinize.hpp)
    for (int k = 0; k < ne; ++k) {
        const double* q = P.elts[k].q[P.stage].data();
        for (int i = 0; i < 3 * nd; ++i)
            if (std::isnan(q[i])) {
                g_err = "Fatal Error: NaN found at element " + std::to_string(P.elts[k].id);
                return 5;
            }
    }
    return 0;
}

}  // namespace

struct orc_handle_s {
    Problem P;
};

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_create(const orc_config* cfg, const orc_mesh* mesh, orc_handle* out) {
    try {
        auto* h = new orc_handle_s();
        build(h->P, cfg, mesh);
        *out = h;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void orc_destroy(orc_handle h) { delete h; }
int64_t orc_n_elements(orc_handle h) { return (int64_t)h->P.elts.size(); }
int32_t orc_ndof(orc_handle h) { return h->P.nd; }

int orc_get_state(orc_handle h, double* q) {
    Problem& P = h->P;
    const int n = 3 * P.nd;
    for (size_t k = 0; k < P.elts.size(); ++k) std::memcpy(q + k * n, P.elts[k].q[P.stage].data(), n * sizeof(double));
    return 0;
}

int orc_set_state(orc_handle h, const double* q) {
    Problem& P = h->P;
    const int n = 3 * P.nd;
    for (size_t k = 0; k < P.elts.size(); ++k) std::memcpy(P.elts[k].q[P.stage].data(), q + k * n, n * sizeof(double));
    return 0;
}

int orc_get_wet(orc_handle h, uint8_t* wet) {
    for (size_t k = 0; k < h->P.elts.size(); ++k) wet[k] = h->P.elts[k].wet ? 1 : 0;
    return 0;
}

int orc_stage(orc_handle h) { return do_stage(h->P); }

int orc_step(orc_handle h, int32_t nsteps) {
    for (int s = 0; s < nsteps; ++s)
        for (int st = 0; st < h->P.ns; ++st) {
            int rc = do_stage(h->P);
            if (rc) return rc;
        }
    return 0;
}

double orc_time(orc_handle h) { return h->P.stage_time(); }

// Simulation::ComputeL2Residual (simulation.hpp:85-93) with Element::ComputeResidualL2 (element.hpp:549-592)
int orc_l2_error(orc_handle h, double* out) {
    Problem& P = h->P;
    const auto& R = P.l2rule;
    const int ng = (int)R.w.size(), nd = P.nd;
    const double t = P.stage_time();
    double total = 0;
    for (auto& E : P.elts) {
        const double* q = E.q[0].data();
        double l2[3] = {0, 0, 0};
        for (int gp = 0; gp < ng; ++gp) {
            double x, y;
            E.shape.local_to_global(R.z1[gp], R.z2[gp], x, y);
            dgsw_fn3 f = dgsw_fn_true(P.cfg.function_set, P.cfg.fn_params, t, x, y);
            double tv[3] = {f.ze, f.qx, f.qy};
            for (int v = 0; v < 3; ++v) {
                double u = 0;
                for (int dof = 0; dof < nd; ++dof) u += q[v * nd + dof] * P.l2phi[dof * ng + gp];
                double d = tv[v] - u;
                l2[v] += (d * d) * R.w[gp];
            }
        }
        double aJ = std::abs(E.shape.detJ());
        double L2 = 0;
        for (int v = 0; v < 3; ++v) L2 += l2[v] * aJ;
        total += L2;
    }
    *out = std::sqrt(total);
    return 0;
}

// total water volume sum_e int_e (ze_h + b_h) dA = sum_e 2 |J| (ze_0 + b_0) (phi_0 = 1, master area 2)
int orc_mass(orc_handle h, double* out) {
    Problem& P = h->P;
    double s = 0;
    for (auto& E : P.elts) s += 2.0 * std::abs(E.detJ) * (E.q[P.stage][0] + E.bath[0]);
    *out = s;
    return 0;
}

int orc_topology(orc_handle h, int32_t* neighbors, uint8_t* btype, int64_t* n_intf, int32_t* intf, int64_t* n_bound,
                 int32_t* bound) {
    Problem& P = h->P;
    for (size_t k = 0; k < P.elts.size(); ++k)
        for (int f = 0; f < 3; ++f) {
            if (neighbors) neighbors[3 * k + f] = P.elts[k].neighbor_idx[f];
            if (btype) btype[3 * k + f] = P.elts[k].btype[f];
        }
    *n_intf = (int64_t)P.intfs.size();
    if (intf)
        for (size_t i = 0; i < P.intfs.size(); ++i) {
            intf[4 * i + 0] = P.intfs[i].in;
            intf[4 * i + 1] = P.intfs[i].ex;
            intf[4 * i + 2] = P.intfs[i].bin;
            intf[4 * i + 3] = P.intfs[i].bex;
        }
    *n_bound = (int64_t)P.bnds.size();
    if (bound)
        for (size_t i = 0; i < P.bnds.size(); ++i) {
            bound[3 * i + 0] = P.bnds[i].elt;
            bound[3 * i + 1] = P.bnds[i].bid;
            bound[3 * i + 2] = P.bnds[i].type;
        }
    return 0;
}

int orc_limited_flags(orc_handle h, uint8_t* flags) {
    for (size_t k = 0; k < h->P.elts.size(); ++k) flags[k] = h->P.elts[k].limited ? 1 : 0;
    return 0;
}

int orc_trouble(orc_handle h, double* I, uint8_t* troubled) {
    for (size_t k = 0; k < h->P.elts.size(); ++k) {
        if (I) I[k] = h->P.elts[k].sl_I;
        if (troubled) troubled[k] = h->P.elts[k].sl_troubled ? 1 : 0;
    }
    return 0;
}

void orc_llf_flux(double g, const double* q_in, const double* q_ex, double bath, double sp, const double* n,
                  double* F) {
    LLF_flux(g, q_in, q_ex, bath, sp, n, F);
}

// ISP::Internal::ComputeFlux at one Gauss point (rkdg_swe_is_internal.hpp:26-95), the per-point body of
// interface_flux above: LLF with the in side's sp, F_ex = -F_in, the wet/dry fix-ups when a side is dry
void orc_internal_flux(double g, const double* qi, const double* qe, double bath_in, double bath_ex, double sp_in,
                       double sp_ex, const double* n, int wet_in, int wet_ex, double* Fi, double* Fe) {
    const double n_in[2] = {n[0], n[1]};
    const double n_ex[2] = {-n[0], -n[1]};
    LLF_flux(g, qi, qe, bath_in, sp_in, n_in, Fi);
    for (int v = 0; v < 3; ++v) Fe[v] = -Fi[v];
    if (Fi[0] > 1e-12) {
        if (!wet_in) {
            for (int v = 0; v < 3; ++v) Fi[v] = 0.0;
            land_flux(g, n_ex, qe, bath_ex, sp_ex, Fe);
        } else if (!wet_ex) {
            LLF_flux(0.0, qe, qi, bath_ex, sp_ex, n_ex, Fe);
            Fe[0] = -Fi[0];
        }
    } else if (Fi[0] < -1e-12) {
        if (!wet_ex) {
            for (int v = 0; v < 3; ++v) Fe[v] = 0.0;
            land_flux(g, n_in, qi, bath_in, sp_in, Fi);
        } else if (!wet_in) {
            LLF_flux(0.0, qi, qe, bath_in, sp_in, n_in, Fi);
            Fi[0] = -Fe[0];
        }
    }
}

// the analytic function sets (true solution / source, bathymetry of Thacker's bowl) at n points, for
// tests that check them against an independent evaluation
int orc_fn_eval(int id, const double* params, double t, int what, int n, const double* x, const double* y,
                double* out) {
    for (int i = 0; i < n; ++i) {
        if (what == 2) {
            out[i] = fn_thacker_bath(params, x[i], y[i]);
            continue;
        }
        const dgsw_fn3 f = what == 1 ? dgsw_fn_source(id, params, t, x[i], y[i]) : dgsw_fn_true(id, params, t, x[i], y[i]);
        out[3 * i] = f.ze;
        out[3 * i + 1] = f.qx;
        out[3 * i + 2] = f.qy;
    }
    return 0;
}

int orc_dubiner(int p, int npt, const double* z1, const double* z2, double* phi, double* dphi1, double* dphi2) {
    vector<double> a(z1, z1 + npt), b(z2, z2 + npt);
    vector<double> ph = get_phi(p, a, b), d1, d2;
    get_dphi(p, a, b, d1, d2);
    std::copy(ph.begin(), ph.end(), phi);
    std::copy(d1.begin(), d1.end(), dphi1);
    std::copy(d2.begin(), d2.end(), dphi2);
    return 0;
}

int orc_triangle_rule(int degree, double* w, double* z1, double* z2, int cap) {
    dgsw::Rule2D r = dgsw::triangle_rule(degree);
    int n = (int)r.w.size();
    for (int i = 0; i < n && i < cap; ++i) {
        w[i] = r.w[i];
        z1[i] = r.z1[i];
        z2[i] = r.z2[i];
    }
    return n;
}

int orc_gl_rule(int degree, double* w, double* z, int cap) {
    dgsw::Rule1D r = dgsw::gauss_legendre_degree(degree);
    int n = (int)r.w.size();
    for (int i = 0; i < n && i < cap; ++i) {
        w[i] = r.w[i];
        z[i] = r.z[i];
    }
    return n;
}

int orc_element_integrals(int p, const double* xy3, int nterm, const double* c, const int* ex, const int* ey,
                          double* integ, double* int_phi, double* int_dphi_x, double* int_dphi_y) {
    Master M;
    M.init(p);
    Shape S;
    for (int v = 0; v < 3; ++v) {
        S.X[v][0] = xy3[2 * v];
        S.X[v][1] = xy3[2 * v + 1];
        S.X[v][2] = 0.0;
    }
    if (S.detJ() < 0) std::swap(S.X[0], S.X[2]);
    double Ji[2][2];
    S.Jinv(Ji);
    double aJ = std::abs(S.detJ());
    const int ngp = M.ngp, nd = M.nd;
    vector<double> f(ngp);
    for (int gp = 0; gp < ngp; ++gp) {
        double x, y;
        S.local_to_global(M.rule.z1[gp], M.rule.z2[gp], x, y);
        double s = 0;
        for (int i = 0; i < nterm; ++i) s += c[i] * std::pow(x, ex[i]) * std::pow(y, ey[i]);
        f[gp] = s;
    }
    double s = 0;
    for (int gp = 0; gp < ngp; ++gp) s += f[gp] * (M.rule.w[gp] * aJ);
    *integ = s;
    for (int dof = 0; dof < nd; ++dof) {
        double a = 0, bx = 0, by = 0;
        for (int gp = 0; gp < ngp; ++gp) {
            a += f[gp] * (M.int_phi[gp * nd + dof] * aJ);
            double dx = 0, dy = 0;
            for (int z = 0; z < 2; ++z) {
                dx += M.int_dphi[z][gp * nd + dof] * Ji[z][0];
                dy += M.int_dphi[z][gp * nd + dof] * Ji[z][1];
            }
            bx += f[gp] * (dx * aJ);
            by += f[gp] * (dy * aJ);
        }
        int_phi[dof] = a;
        int_dphi_x[dof] = bx;
        int_dphi_y[dof] = by;
    }
    return nd;
}

int orc_wet_dry_single(const double* xy3, const double* bath_vrtx, double h_o, const double* q_vrtx_in, int wet_in,
                       double* q_vrtx_out, int* wet_out) {
    // the unit test builds q by L2ProjectionNode of vertex values, runs the kernel, and reads the
    // vertex values back through ProjectBasisToLinear (test_wetting_drying.cpp)
    Master M;
    M.init(1);
    Shape S;
    for (int v = 0; v < 3; ++v) {
        S.X[v][0] = xy3[2 * v];
        S.X[v][1] = xy3[2 * v + 1];
        S.X[v][2] = 0.0;
    }
    double aJ = std::abs(S.detJ());
    const int ngp = M.ngp, nd = M.nd;
    double q[9];
    for (int var = 0; var < 3; ++var) {
        vector<double> a(ngp);
        for (int gp = 0; gp < ngp; ++gp) {
            double ps[3];
            Shape::psi(M.rule.z1[gp], M.rule.z2[gp], ps);
            double s = 0;
            for (int n = 0; n < 3; ++n) s += q_vrtx_in[var * 3 + n] * ps[n];
            a[gp] = s;
        }
        for (int dof = 0; dof < nd; ++dof) {
            double s = 0;
            for (int gp = 0; gp < ngp; ++gp) s += a[gp] * (M.int_phi[gp * nd + dof] * aJ);
            q[var * nd + dof] = s * (M.minv[dof] / aJ);
        }
    }
    double bmin = std::min(bath_vrtx[0], std::min(bath_vrtx[1], bath_vrtx[2]));
    bool wet = wet_in != 0;
    wetting_drying(M, h_o, 1.0e6 * h_o * DBL_EPS, bath_vrtx, bmin, q, wet);
    double ql[3][3];
    M.basis_to_linear(q, ql);
    for (int var = 0; var < 3; ++var)
        for (int v = 0; v < 3; ++v) q_vrtx_out[var * 3 + v] = ql[var][v];
    *wet_out = wet ? 1 : 0;
    return 0;
}

int orc_rk_table(int nstages, int order, double* ark, double* brk, double* drk) {
    dgsw_rk_table T;
    if (dgsw_rk_table_init(nstages, order, &T) != 0) return -1;
    for (int i = 0; i < nstages; ++i) {
        drk[i] = T.drk[i];
        for (int j = 0; j < nstages; ++j) {
            ark[i * nstages + j] = T.ark[i][j];
            brk[i * nstages + j] = T.brk[i][j];
        }
    }
    return 0;
}

}  // extern "C"
