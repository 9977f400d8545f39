// Host-side preprocessing of the RKDG library: mesh topology in the reference's order, the element
// permutation and CTA tiling used on the device, per-tile edge lists, master tables and the FP64
// initial projections. Host C++ only.
#ifndef DGSW_HOST_SETUP_H
#define DGSW_HOST_SETUP_H

#include <cstdint>
#include <memory>
#include <utility>
#include <string>
#include <vector>

#include "../../include/dgsw_rkdg.h"

namespace dgsw {

// allocator whose value-less construct leaves elements uninitialised: large set-up arrays that are
// written in full by parallel loops skip the serial zero fill of std::vector::resize
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) {}
    template <typename U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using bigvec = std::vector<T, UninitAlloc<T>>;

constexpr int MAX_ND = 6;  // p <= 2
constexpr int MAX_NQ = 6;
constexpr int MAX_NG = 3;

// Edge kinds in the per-tile edge lists
enum EdgeKind { EK_INTERIOR = 0, EK_LAND = 1, EK_FUNCTION = 2, EK_TIDE = 3, EK_FLOW = 4, EK_LEVEE = 5 };

struct Topology {
    int64_t ne = 0, nn = 0;
    std::vector<uint32_t> ids;      // reference element IDs, ascending
    std::vector<int32_t> src;       // caller index of element r
    std::vector<int32_t> enodes;    // [3*ne] node indices of element r
    std::vector<int32_t> nbr;       // [3*ne] neighbor element (reference order) or -1
    std::vector<int8_t> nbr_face;   // [3*ne] neighbor's local face or -1
    std::vector<uint8_t> btype;     // [3*ne] DGSW_BC_* (128 interior)
    bigvec<int32_t> intf;           // [4*n_intf] in, ex, face_in, face_ex in creation order
    int64_t n_intf_internal = 0;    // the internal interfaces come first, then the levee ones
    std::vector<int32_t> bnd;       // [3*n_bnd] elem, face, type in traversal order
    // per element: faces in accumulation order (interfaces by creation order, then boundaries)
    std::vector<uint8_t> order_count;  // [ne]
    std::vector<uint8_t> order_face;   // [3*ne]
    std::vector<uint8_t> is_in;        // [3*ne] element is the "in" side of the interface on this face
    // ensembles: member of element r (empty for a single problem) and each member's function-set
    // parameters [n_members][DGSW_FN_PARAMS]
    std::vector<int32_t> group;
    std::vector<double> group_params;
    // tide / flow boundaries: forcing record of boundary i (T.bnd order), -1 for the other types
    std::vector<int32_t> bnd_force;
};

// Tide and flow forcing of the boundary faces (BC::Tide / BC::Flow constructors and Initialize,
// discretization_RKDG/boundary_conditions/rkdg_swe_bc_tide.hpp:33-71): one record per forced face, in
// T.bnd order, holding its first constituent entry and their count; per entry the frequency, forcing
// factor and equilibrium argument, then amplitude and phase at the edge Gauss points.
constexpr int FORCE_STRIDE = 3 + 2 * MAX_NG;
struct Forcing {
    std::vector<int32_t> face;  // [2 * n_forced] first entry, n_constituents
    std::vector<double> con;    // [FORCE_STRIDE * n_entries]: freq, forcing_fact, equilib_arg, amp[NG], phase[NG]
};

// matches tide/flow faces to their .bcis blocks (create_boundaries, swe_pre_create_bound.hpp:33-96) and
// interpolates amplitude and phase to the face's Gauss points; fills T.bnd_force
int build_forcing(const dgsw_mesh* m, Topology& T, int p, Forcing& out, std::string& err);

// Levee interfaces (ISP::Levee constructor + Initialize, rkdg_swe_is_levee.hpp:36-62): per levee interface
// (T.intf from n_intf_internal on) the in face's outward normal, then crest height, subcritical and
// supercritical coefficients at the edge Gauss points (in side order) from the .bcis pairs of its nodes
// (swe_pre_create_intface.hpp:50-66), then the spherical correction at the in side's and at the ex side's
// Gauss points (each in its own order)
constexpr int LEVEE_STRIDE = 2 + 5 * MAX_NG;
int build_levees(const dgsw_mesh* m, const Topology& T, int p, const double* node_xyz, const dgsw_config& cfg,
                 std::vector<double>& out, std::string& err);

// Manning friction: per element g * (mean of its three nodes' n)^2 (swe_pre_init_data.hpp:165-196),
// in reference element order
void manning_factor(const Topology& T, const double* node_n, double g, std::vector<double>& out);

// reference MeshMetaData + create_interfaces/create_boundaries semantics
int build_topology(const dgsw_mesh* m, Topology& T, std::string& err);

struct Tiling {
    int tile = 256;
    int64_t ntiles = 0;
    std::vector<int32_t> dev_of_ref;  // [ne]
    std::vector<int32_t> ref_of_dev;  // [ne]
    std::vector<int32_t> tile_edge_off;  // [ntiles+1]
    // [4 * n_edges]: trace slot of the in/owner side a, trace slot of b (-1 for boundaries),
    // meta = face_a | face_b << 2 | kind << 4, device index of a. Trace slots: 3*(element - tile start)
    // + face for tile elements, 3*tile + h for the tile's halo face h.
    bigvec<int32_t> edges;
    bigvec<double> egeo;                 // [3 * n_edges]: normal x, normal y, half length (of face a)
    std::vector<int32_t> tile_halo_off;  // [ntiles+1]
    bigvec<int32_t> halo;                // [2 * n_halo]: device element, face
    std::vector<int32_t> eslot;          // [2 * ne] per element (dev order): packed slots, roles + order
    int max_edges = 0;
    int max_halo = 0;
};

int build_tiling(const Topology& T, const double* node_xyz, int tile, bool morton, Tiling& out, std::string& err);

// Master-element tables in the layouts the kernels read
struct Tables {
    int p = 1, nd = 3, nq = 3, ng = 2;
    double phi[MAX_ND * MAX_NQ];         // [dof][gp]
    double dphi[2][MAX_ND * MAX_NQ];     // [z][dof][gp]
    double mz[2][MAX_NQ * MAX_ND];       // [z][gp][dof] = dphi_z(dof,gp) * w(gp)
    double phiw[MAX_NQ * MAX_ND];        // [gp][dof]   = phi(dof,gp) * w(gp)
    double psi[3][MAX_NQ];               // nodal (linear) shape functions at the volume points
    double w[MAX_NQ];
    double fphi[3][MAX_ND * MAX_NG];     // [face][dof][gp]
    double fpsi[3][3][MAX_NG];           // [face][node][gp]
    double gw[MAX_NG];
    double minv[MAX_ND];
};

int build_tables(int p, Tables& t, std::string& err);

// Dubiner modes of order p at n master points: phi[dof * n + pt]
void eval_basis(int p, const double* z1, const double* z2, int n, double* phi);

// element geometry in the reference's formulas (shape_straighttriangle.cpp:95-137):
// J^-1(0,0), J^-1(0,1), J^-1(1,0), J^-1(1,1), |det J|
void element_geometry(const double* node_xyz, const int32_t* nodes3, double out[5]);
// outward unit normal and surface Jacobian (half length) of face f (shape_straighttriangle.cpp:110-168)
void face_geometry(const double* node_xyz, const int32_t* nodes3, int f, double& nx, double& ny, double& sJ);

// FP64 host projections of initialize_data_serial: bathymetry modes per element (reference order)
void project_bathymetry(const Topology& T, const double* node_xyz, const Tables& tb, std::vector<double>& bath);
// initial condition modes [ne][3][nd] (reference order)
void project_initial_condition(const Topology& T, const double* node_xyz, const Tables& tb, const dgsw_config& cfg,
                               std::vector<double>& q);
// wetting/drying initialisation on the projected state (swe_pre_init_data.hpp:213-250); returns wet flags
void init_wet_dry(const Topology& T, const double* node_xyz, const Tables& tb, const dgsw_config& cfg,
                  std::vector<double>& q, std::vector<uint8_t>& wet);

}  // namespace dgsw

#endif
