// CPU FP64 oracle for the dgswemv2 RKDG shallow-water step.
//
// TEST INFRASTRUCTURE ONLY. This is a restatement, in plain C++, of the reference's serial RKDG
// path (source/problem/SWE/discretization_RKDG/kernels_processor/rkdg_swe_proc_serial_step.hpp:29-67)
// with the reference's data layout semantics (per-element precomputed integration factors,
// element.hpp:167-272), traversal order (elements by ascending ID, interfaces in (in_id, ex_id)
// creation order, boundaries grouped by condition type) and accumulation order. It exists to check
// the CUDA library; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
//
// Parity anchor: the reference itself cannot be compiled in this environment (it needs Eigen,
// yaml-cpp and METIS, none of which are present), so this oracle is pinned against the golden
// vectors the reference's own unit tests hold (tests/golden/, generated from test/*.cpp).
#ifndef DGSW_ORACLE_HPP
#define DGSW_ORACLE_HPP

#include <cstdint>

extern "C" {

// problem description shared with the C ABI of the library (same field meaning)
struct orc_config {
    int32_t p;
    int32_t rk_nstages, rk_order;
    double dt;
    double g;
    int32_t wetting_drying;
    double h_o;
    int32_t slope_limiting;
    double sl_M, sl_nu;
    int32_t function_source;
    int32_t ic_type;      // 0 default/constant, 1 function
    double ic_const[3];   // ze, qx, qy for constant initial conditions
    int32_t function_set; // see function_sets.h
    double fn_params[16];
    int32_t spherical;    // spherical projection on/off
    double sp_lat0_deg, sp_R;
    int32_t n_threads;    // OpenMP threads for the element/edge sweeps (1 = serial)
    int32_t bottom_friction;  // 0 none, 1 Chezy, 2 Manning (swe_definitions.hpp:92)
    double friction_cf;       // bottom_friction.coefficient
    double ramp_duration;     // timestepping.ramp_duration (days)
};

// one tide / flow block of the .bcis file (read_bcis, swe_inputs.cpp:211-290)
struct orc_forcing_block {
    int32_t type;  // 1 tide, 2 flow
    int32_t n_nodes;
    int32_t n_constituents;
    const int32_t* nodes;        // [n_nodes] node indices
    const double* frequency;     // [n_constituents]
    const double* forcing_fact;  // [n_constituents]
    const double* equilib_arg;   // [n_constituents]
    const double* amplitude;     // [n_constituents][n_nodes]
    const double* phase;         // [n_constituents][n_nodes]
};

// mesh: node coordinates (x,y,z = bathymetry depth), element node triples (0-based node indices,
// reference element IDs optional), boundary segments as ADCIRC-style node chains with a type
// (0 land, 1 tide, 2 flow, 3 function, 4 outflow).
struct orc_mesh {
    int64_t n_nodes;
    const double* node_xyz;
    int64_t n_elems;
    const int32_t* elem_nodes;
    const uint32_t* elem_ids;  // may be null: IDs 0..n_elems-1
    int32_t n_segments;
    const int32_t* seg_type;
    const int64_t* seg_offsets;  // n_segments+1
    const int32_t* seg_nodes;
    const double* node_manning_n;  // [n_nodes] Manning's n (bottom_friction 2), or null
    int32_t n_forcing;
    const orc_forcing_block* forcing;
    // internal barriers: a segment of type 129 holds n front nodes then n back nodes; the .bcis levee
    // lines give (front, back) pairs with H_barrier, C_subcritical, C_supercritical
    int32_t n_levee_pairs;
    const int32_t* levee_nodes;  // [2 * n_levee_pairs]
    const double* levee_data;    // [3 * n_levee_pairs]
};

typedef struct orc_handle_s* orc_handle;

int orc_create(const orc_config* cfg, const orc_mesh* mesh, orc_handle* out);
void orc_destroy(orc_handle h);
const char* orc_last_error(void);

int64_t orc_n_elements(orc_handle h);
int32_t orc_ndof(orc_handle h);
// state in ascending element-ID order, layout [elem][var][dof]
int orc_get_state(orc_handle h, double* q);
int orc_set_state(orc_handle h, const double* q);
int orc_get_wet(orc_handle h, uint8_t* wet);
int orc_step(orc_handle h, int32_t nsteps);
int orc_stage(orc_handle h);
double orc_time(orc_handle h);
int orc_l2_error(orc_handle h, double* out);
int orc_mass(orc_handle h, double* out);
// topology in ascending element-ID order: neighbor element index (-1 none), boundary type per face
// (255 internal), the interface list (in elem index, ex elem index, in face, ex face) in creation order
// and the boundary list (elem index, face, type) in traversal order
int orc_topology(orc_handle h, int32_t* neighbors, uint8_t* btype, int64_t* n_intf, int32_t* intf,
                 int64_t* n_bound, int32_t* bound);
// limiter decision of the last limiter pass: 1 if the element's state was changed
int orc_limited_flags(orc_handle h, uint8_t* flags);
// per-element KXRCF trouble indicator of the last limiter pass (swe_trouble_check.hpp)
int orc_trouble(orc_handle h, double* I, uint8_t* troubled);

// unit-level entry points used to pin the oracle against the reference's unit-test vectors
void orc_llf_flux(double g, const double* q_in, const double* q_ex, double bath, double sp, const double* n,
                  double* F);
// ISP::Internal::ComputeFlux at one Gauss point (LLF, F_ex = -F_in, wet/dry fix-ups for a dry side)
void orc_internal_flux(double g, const double* qi, const double* qe, double bath_in, double bath_ex, double sp_in,
                       double sp_ex, const double* n, int wet_in, int wet_ex, double* Fi, double* Fe);
// function set `id` at n points: what 0 = true solution, 1 = source (out [n][3]), 2 = Thacker bathymetry (out [n])
int orc_fn_eval(int id, const double* params, double t, int what, int n, const double* x, const double* y,
                double* out);
int orc_dubiner(int p, int npt, const double* z1, const double* z2, double* phi, double* dphi1, double* dphi2);
int orc_triangle_rule(int degree, double* w, double* z1, double* z2, int cap);
int orc_gl_rule(int degree, double* w, double* z, int cap);
// integrals of gp values over an element of master order p (element.hpp Integration / IntegrationPhi /
// IntegrationDPhi); f is evaluated at the element's own gp global coordinates by the caller-supplied
// polynomial coefficients c: f = sum c[i] x^ex[i] y^ey[i]
int orc_element_integrals(int p, const double* xy3, int nterm, const double* c, const int* ex, const int* ey,
                          double* integ, double* int_phi, double* int_dphi_x, double* int_dphi_y);
// single-element wetting/drying kernel (swe_post_wet_dry.hpp) on a p=1 element: vertex values in,
// vertex values and wet flag out
int orc_wet_dry_single(const double* xy3, const double* bath_vrtx, double h_o, const double* q_vrtx_in,
                       int wet_in, double* q_vrtx_out, int* wet_out);
int orc_rk_table(int nstages, int order, double* ark, double* brk, double* drk);
}

#endif
