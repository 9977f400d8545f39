/* dgsw_rkdg.h - C ABI of the B200 RKDG shallow-water library (libdgsw_rkdg.so).
 *
 * The library replaces the serial RKDG step of dgswemv2 behind the reference's problem/stepper
 * interface SWE::RKDG::Problem (source/problem/SWE/discretization_RKDG/rkdg_swe_problem.hpp:34-194).
 * Each entry point below names the reference interface it stands in for. Plain C types only: the
 * caller owns every host array (copied in at create/set, copied out at get); the library owns the
 * device buffers, its CUDA stream and its CUDA graphs.
 *
 * Errors: every function returns a dgsw_status; 0 is success. A failing call leaves a message that
 * dgsw_last_error() returns (per host thread). Nothing aborts or traps: the reference's abort() on a
 * NaN (rkdg_swe_proc_serial_step.hpp:59-65) becomes DGSW_ERR_NAN from dgsw_rkdg_step.
 * Threading: one host thread per handle at a time; all work is ordered on the handle's stream.
 */
#ifndef DGSW_RKDG_H
#define DGSW_RKDG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGSW_ABI_VERSION 3
#define DGSW_TILE_AUTOTUNE (-1)

typedef enum {
    DGSW_OK = 0,
    DGSW_ERR_INVALID_ARGUMENT = 1,
    DGSW_ERR_MESH = 2,          /* topology / boundary lookup errors (std::logic_error in the reference) */
    DGSW_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    DGSW_ERR_NAN = 4,           /* NaN in the modal state after a stage (scrutinize_solution) */
    DGSW_ERR_UNSUPPORTED = 5,   /* a feature of the input this build does not implement */
    DGSW_ERR_NO_DEVICE = 6,     /* no CUDA device visible */
    DGSW_ERR_IO = 7             /* input file could not be read or parsed */
} dgsw_status;

typedef enum { DGSW_FP64 = 0, DGSW_FP32 = 1 } dgsw_precision;

/* Bottom friction types, source/problem/SWE/swe_definitions.hpp:92 */
enum { DGSW_FRICTION_NONE = 0, DGSW_FRICTION_CHEZY = 1, DGSW_FRICTION_MANNING = 2 };

/* Boundary condition / edge types, source/problem/SWE/swe_definitions.hpp:61-69 */
enum { DGSW_BC_LAND = 0, DGSW_BC_TIDE = 1, DGSW_BC_FLOW = 2, DGSW_BC_FUNCTION = 3, DGSW_BC_OUTFLOW = 4,
       DGSW_BC_INTERNAL = 128, DGSW_BC_LEVEE = 129 };

/* Problem configuration: the `.15` input surface read by InputParameters
 * (source/preprocessor/input_parameters.hpp:95-261) and SWE::Inputs (problem_input/swe_inputs.cpp:4-205)
 * that the RKDG step consumes, plus the B200-specific execution options at the end. */
typedef struct {
    int32_t p;                 /* polynomial_order (1 or 2) */
    int32_t rk_nstages;        /* timestepping.nstages */
    int32_t rk_order;          /* timestepping.order */
    double dt;                 /* timestepping.dt */
    double g;                  /* problem.gravity */
    int32_t wetting_drying;    /* problem.wetting_drying present */
    double h_o;                /* problem.wetting_drying.h_o */
    int32_t slope_limiting;    /* problem.slope_limiting.type == Cockburn-Shu */
    double sl_M, sl_nu;        /* problem.slope_limiting.{M,nu} */
    int32_t function_source;   /* problem.function_source: Enable */
    int32_t ic_type;           /* problem.initial_conditions.type: 0 Default/Constant, 1 Function */
    double ic_const[3];        /* initial_surface_height, initial_momentum_x, initial_momentum_y */
    int32_t function_set;      /* which ic_q/source_q/true_q set (function_sets.h) */
    double fn_params[16];      /* parameters of that set */
    int32_t spherical;         /* problem.spherical_projection present */
    double sp_lat0_deg, sp_R;  /* spherical_projection.{latitude_o, R} */
    int32_t bottom_friction;   /* problem.bottom_friction.type: DGSW_FRICTION_{NONE,CHEZY,MANNING} */
    double friction_cf;        /* bottom_friction.coefficient: Chezy Cf, or the lower bound of the Manning
                                  factor g n^2 / h^(1/3) */
    double ramp_duration;      /* timestepping.ramp_duration in days (tide/flow forcing ramp; 0 = none) */
    /* execution options (no reference counterpart) */
    int32_t precision;         /* dgsw_precision: FP64, or FP32 bulk arithmetic (volume, edge and source
                                  integrals) with FP64 stage states, wet/dry tests, limiter and reductions */
    int32_t device;            /* CUDA device ordinal */
    int32_t tile;              /* elements per stage-kernel tile: 128 or 256; 0 = 128; DGSW_TILE_AUTOTUNE =
                                  time every (tile, occupancy, tile_order) candidate on the device at create
                                  and keep the fastest (dgsw_rkdg_tuning reports the timings) */
    int32_t renumber;          /* 0 keep input order, 1 Morton order of element centroids (default 1) */
    int32_t use_graphs;        /* capture each RK step in a CUDA graph (default 1) */
    int32_t fp64_limiter;      /* FP32 precision only: 1 runs the slope limiter's characteristic arithmetic in
                                  FP64; 0 (default) in FP32 on FP64 differences, with the write-back test
                                  free of FP32 rounding (limiter_kernel.cuh) */
    int32_t occupancy;         /* stage-kernel register budget: 0 the default resident CTAs per SM, 1 the
                                  alternative (one CTA fewer, or one more where the default is one); set by
                                  the autotuner when tile = DGSW_TILE_AUTOTUNE */
    int32_t tile_order;        /* 0 alternate the tile order from stage to stage (each stage starts where
                                  the previous one ended), 1 always ascending; set by the autotuner too */
    int32_t fp64_stages;       /* FP32 precision only: 1 keeps every intermediate stage state in FP64; 0
                                  (default) keeps them as FP32 increments from the carried state, itself
                                  kept as two FP32 parts (q_s = q_0 + d_s; q_0 + d_ns is formed in FP64 at each
                                  step's last stage) wherever only the stage kernel reads them: without
                                  wetting/drying, slope limiter or levees, and with three or more stages */
    int32_t reserved[4];
} dgsw_config;

/* One tide or flow block of the `.bcis` file (SWE::Inputs::read_bcis, problem_input/swe_inputs.cpp:211-
 * 290): its nodes and, per constituent, frequency (rad/s), forcing factor and equilibrium argument
 * (degrees), and the amplitude and phase (degrees) at each node. A tide/flow boundary face takes its data
 * from the first block of its type that holds both of its nodes (create_boundaries,
 * problem_preprocessor/swe_pre_create_bound.hpp:33-96). */
typedef struct {
    int32_t type;              /* DGSW_BC_TIDE or DGSW_BC_FLOW */
    int32_t n_nodes;
    int32_t n_constituents;
    const int32_t* nodes;      /* [n_nodes] 0-based node indices, each at most once */
    const double* frequency;   /* [n_constituents] */
    const double* forcing_fact;
    const double* equilib_arg;
    const double* amplitude;   /* [n_constituents][n_nodes] */
    const double* phase;       /* [n_constituents][n_nodes] */
} dgsw_forcing_block;

/* Mesh: node coordinates (x, y, bathymetry depth), element node triples (0-based node indices), the
 * reference element IDs (the order the reference iterates elements in; NULL = 0..n-1), and ADCIRC-style
 * boundary node chains with their types, searched in the given order like AdcircFormat::get_ibtype
 * (source/preprocessor/ADCIRC_reader/adcirc_format.cpp:214-259), then the optional Manning and tide/flow
 * data. A DGSW_BC_LEVEE chain is an ADCIRC internal barrier (IBTYPE % 10 == 4, :89-102): its n front
 * nodes (NBVV) followed by its n back nodes (IBCONN), so 2n entries; the faces along either side become
 * levee interfaces to the element across the barrier (MeshMetaData, mesh_metadata.cpp:65-83), with the
 * crest height and the sub- / supercritical discharge coefficients of the .bcis levee lines
 * (levee_nodes: front, back per pair; levee_data: H_barrier, C_subcritical, C_supercritical per pair;
 * swe_inputs.cpp:274-287, swe_pre_create_intface.hpp:38-78). */
typedef struct {
    int64_t n_nodes;
    const double* node_xyz;     /* [3*n_nodes] */
    int64_t n_elems;
    const int32_t* elem_nodes;  /* [3*n_elems] */
    const uint32_t* elem_ids;   /* [n_elems] or NULL */
    int32_t n_segments;
    const int32_t* seg_type;    /* [n_segments], DGSW_BC_* */
    const int64_t* seg_offsets; /* [n_segments+1] */
    const int32_t* seg_nodes;   /* [seg_offsets[n_segments]] */
    const double* node_manning_n;        /* [n_nodes] Manning's n per node (DGSW_FRICTION_MANNING), or NULL */
    int32_t n_forcing;                   /* tide / flow forcing blocks */
    const dgsw_forcing_block* forcing;   /* [n_forcing] */
    int32_t n_levee_pairs;               /* .bcis levee lines */
    const int32_t* levee_nodes;          /* [2 * n_levee_pairs] front, back node indices */
    const double* levee_data;            /* [3 * n_levee_pairs] H_barrier, C_subcritical, C_supercritical */
} dgsw_mesh;

typedef struct {
    int64_t n_elems, n_nodes, n_interfaces, n_boundaries, n_tiles, n_tile_edges;
    int32_t p, ndof, ngp_volume, ngp_edge, nstages, precision, tile;
    int64_t device_bytes;      /* bytes of device memory held by the handle */
    int64_t state_bytes;       /* bytes of one stage state array */
    int32_t occupancy, tile_order;  /* the stage kernel's register budget and tile order in use */
    int32_t stage_increments;  /* 1 when the intermediate stage states are FP32 increments (fp64_stages) */
    int32_t smem_capped;       /* 1 when the stage kernel's shared memory has the compile-time capacities;
                                  0 when it is sized to the mesh's largest tile (the autotuner's choice, or a
                                  tile beyond the capacities) */
} dgsw_info;

typedef struct dgsw_rkdg_s* dgsw_handle;

/* library -------------------------------------------------------------------------------------- */
int32_t dgsw_abi_version(void);
const char* dgsw_last_error(void);
const char* dgsw_status_string(int32_t status);
void dgsw_config_default(dgsw_config* cfg);

/* Problem::initialize_problem_parameters + preprocess_mesh_data + create_interfaces/boundaries +
 * Simulation ctor (rkdg_swe_problem.hpp:55-92, simulation.hpp:36-65, initialize_mesh.hpp:19-77):
 * builds topology, interface/boundary order and device geometry. Does not set the state. */
int32_t dgsw_rkdg_create(const dgsw_config* cfg, const dgsw_mesh* mesh, dgsw_handle* out);
int32_t dgsw_rkdg_destroy(dgsw_handle h);

/* Ensemble batching (no counterpart in the reference, which runs one mesh per process): n_members
 * independent problems that share one configuration (order, RK method, dt, wetting/drying, limiter,
 * precision) but each have their own mesh, bathymetry and initial-condition parameters
 * (member_params: [n_members][16] values of the configuration's function set, NULL = cfg->fn_params for
 * all; sources and function boundaries use cfg->fn_params). All members advance together: one
 * stage-kernel launch per RK stage covers every member, and dgsw_rkdg_step replays one CUDA graph per
 * step. The handle behaves like any other: the state and wet flags are laid out member after member
 * (member k's elements in ascending order of its own element IDs), see dgsw_ensemble_member_range.
 * With cfg->tile == DGSW_TILE_AUTOTUNE the tile size is tuned on the leading members (about 2^19
 * elements). */
int32_t dgsw_ensemble_create(const dgsw_config* cfg, int32_t n_members, const dgsw_mesh* members,
                             const double* member_params, dgsw_handle* out);
/* element range of one member in the handle's state order (a single problem is member 0) */
int32_t dgsw_ensemble_member_range(dgsw_handle h, int32_t member, int64_t* first, int64_t* n_elems);
/* the autotuner's record, one entry per timed candidate: tile size, occupancy, tile order and device
 * milliseconds per step (*n = 0 when the handle was not tuned, or reused a cached decision). Pass NULL
 * arrays to query *n; otherwise the arrays hold at least DGSW_TUNE_MAX_CANDIDATES entries. */
#define DGSW_TUNE_MAX_CANDIDATES 8
int32_t dgsw_rkdg_tuning(dgsw_handle h, int32_t* tiles, int32_t* occupancy, int32_t* tile_order, double* ms_per_step,
                         int32_t* n);
int32_t dgsw_rkdg_info(dgsw_handle h, dgsw_info* out);

/* Problem::preprocessor_serial -> initialize_data_serial (swe_pre_init_data.hpp:9-327): bathymetry and
 * initial-condition L2 projections, wetting/drying and limiter initialisation; resets time to 0. */
int32_t dgsw_rkdg_init_state(dgsw_handle h);

/* modal state of the current stage in ascending element-ID order, layout [elem][var(ze,qx,qy)][dof],
 * FP64 on the host (elt.data.state[stage].q, swe_data_state.hpp:5-17). set_state leaves wet flags as
 * they are; call dgsw_rkdg_set_wet to change them. */
int32_t dgsw_rkdg_set_state(dgsw_handle h, const double* q);
int32_t dgsw_rkdg_get_state(dgsw_handle h, double* q);
/* Output values for the VTK / VTU writers (write_VTK_data / write_VTU_data,
 * problem_postprocessor/swe_post_write_vtk.hpp:5-95, swe_post_write_vtu.hpp:5-104, N_DIV = 1), evaluated
 * from the current state on the device, in ascending element-ID order: point_data [n_elems][3 vertices]
 * [ze, qx, qy, bath], cell_data [n_elems][ze, qx, qy, bath] at the centroid, the wet flags and the
 * went-completely-dry flags of the last wet/dry pass (wet and went_dry may be NULL). */
int32_t dgsw_rkdg_postprocess(dgsw_handle h, double* point_data, double* cell_data, uint8_t* wet, uint8_t* went_dry);
/* the bathymetry's modal L2 projection (state[0].aux, swe_pre_init_data.hpp:22-25), [n_elems][ndof] in
 * ascending element-ID order, as the modal writer prints it (host computation, no device work) */
int32_t dgsw_rkdg_get_bathymetry(dgsw_handle h, double* modes);
int32_t dgsw_rkdg_set_wet(dgsw_handle h, const uint8_t* wet);
int32_t dgsw_rkdg_get_wet(dgsw_handle h, uint8_t* wet);
/* the same on device buffers of the library's device (layout [elem][var][dof], FP64 in both precisions:
 * the FP32 path computes in FP32 but keeps its stage states in FP64); ordered on the handle's stream */
int32_t dgsw_rkdg_set_state_device(dgsw_handle h, const void* d_q);
int32_t dgsw_rkdg_get_state_device(dgsw_handle h, void* d_q);

/* Problem::step_serial / stage_serial (rkdg_swe_proc_serial_step.hpp:10-67): advance nsteps full RK
 * steps (or one stage). Returns DGSW_ERR_NAN if a NaN appeared (checked once at the end of the call). */
int32_t dgsw_rkdg_step(dgsw_handle h, int32_t nsteps);
int32_t dgsw_rkdg_stage(dgsw_handle h);
/* ESSPRKStepper::GetTimeAtCurrentStage / GetStep / GetStage (explicit_ssp_rk_stepper.hpp:42-46) */
int32_t dgsw_rkdg_get_time(dgsw_handle h, double* t, int64_t* step, int32_t* stage);

/* Simulation::ComputeL2Residual (simulation.hpp:85-93): sqrt of the sum over elements of
 * int (true_q(t) - q_h)^2 over ze, qx, qy, on the device in FP64 */
int32_t dgsw_rkdg_l2_error(dgsw_handle h, double* out);
/* total water volume sum_e int_e (ze_h + b_h) dA, FP64 device reduction (no reference counterpart;
 * the global mass balance check of the FP32 path) */
int32_t dgsw_rkdg_mass(dgsw_handle h, double* out);

/* Allocation-free L2 error of a caller-owned FP64 state; no counterpart in the reference.
 * For callers that may not allocate device memory during a run: drivers whose memory pool (PyTorch's
 * caching allocator, a coupler's arena) already holds the GPU's memory, and monitoring code between
 * asynchronously queued steps, where cudaMalloc/cudaFree can synchronise the device. It calls no
 * cudaMalloc, cudaFree or other allocating routine and needs no handle; its scratch is a fixed static
 * device array of 32 KiB per device, so n_elems is limited to DGSW_L2_STATIC_MAX_ELEMS (larger inputs
 * are rejected with DGSW_ERR_INVALID_ARGUMENT; dgsw_rkdg_l2_error has no such limit).
 * Same value as dgsw_rkdg_l2_error up to summation order. Inputs, all on the current device:
 * d_q [n_elems][3][ndof] FP64 (the layout dgsw_rkdg_get_state_device writes),
 * d_elem_nodes [n_elems][3] 0-based node indices, d_node_xyz [n_nodes][3] (x, y, depth);
 * function_set / fn_params (16 values, NULL = zeros) / t select true_q. Work is queued on `stream`
 * (NULL = default stream) and the call returns after it completes, with the result in *out (host).
 * The first call on a device does a one-time set-up (copies the quadrature table to the device and
 * looks up the scratch address); make that first call before any stream capture. The set-up is kept
 * for the life of the process, so a cudaDeviceReset between calls is not supported (the saved address and
 * the device-side table would be stale). All calls on one device share the scratch array: calls that
 * overlap on the GPU race and may return wrong values. */
#define DGSW_L2_STATIC_MAX_ELEMS 1048576
int32_t dgsw_l2_error_static(int32_t p, int64_t n_elems, const double* d_q, const int32_t* d_elem_nodes,
                             const double* d_node_xyz, int32_t function_set, const double* fn_params, double t,
                             void* stream, double* out);

/* integer topology in ascending element-ID order, for bit-exact comparison with the reference's
 * MeshMetaData (mesh_metadata.cpp:3-85) and interface/boundary creation (swe_pre_create_intface.hpp,
 * swe_pre_create_bound.hpp): neighbor element index per face (-1 none), boundary type per face
 * (DGSW_BC_INTERNAL for interior faces), interfaces (in, ex, face_in, face_ex) in creation order,
 * boundaries (elem, face, type) in traversal order. Pass NULL arrays to query the counts. */
int32_t dgsw_rkdg_topology(dgsw_handle h, int32_t* neighbors, uint8_t* btype, int64_t* n_interfaces,
                           int32_t* interfaces, int64_t* n_boundaries, int32_t* boundaries);

/* The same topology computed on the host only (no device needed): MeshMetaData + interface and
 * boundary creation for a mesh. Arrays as for dgsw_rkdg_topology; pass NULL to query counts. */
int32_t dgsw_mesh_topology(const dgsw_mesh* mesh, int32_t* neighbors, uint8_t* btype, int64_t* n_interfaces,
                           int32_t* interfaces, int64_t* n_boundaries, int32_t* boundaries);

/* check_trouble (swe_trouble_check.hpp:6-116): the KXRCF-type indicator the reference evaluates in every
 * limiter pass but does not use. Off by default; once enabled, each limiter pass also computes it on the
 * state the limiter sees, and dgsw_rkdg_get_trouble returns the last pass's indicator I and troubled
 * flags (after the five-layer neighbour growth), in ascending element-ID order (either may be NULL). */
int32_t dgsw_rkdg_set_trouble(dgsw_handle h, int32_t enable);
int32_t dgsw_rkdg_get_trouble(dgsw_handle h, double* I, uint8_t* troubled);

/* per element 1 if the last slope-limiter pass changed its state (the plain limiter's decision) */
int32_t dgsw_rkdg_get_limited(dgsw_handle h, uint8_t* flags);

/* ---- learned troubled-cell indicator (no counterpart in the reference) ----------------------------
 * An 18 -> 64 -> 64 -> 1 MLP (ReLU, sigmoid) predicts whether the Cockburn-Shu limiter
 * (CS_slope_limiter_serial, swe_CS_sl_serial.hpp:9-23) will change a cell, from the cell's linear modal
 * coefficients and its neighbours' means, scaled per field (18 features; p = 1 only). Parameters: FP32,
 * DGSW_MLP_NPARAM values laid out W1[64][18], b1[64], W2[64][64], b2[64], w3[64], b3. Inference runs on the
 * tensor cores (BF16 inputs and weights, FP32 accumulation); training runs in FP32. */
#define DGSW_MLP_NPARAM 5441
#define DGSW_MLP_NFEATURES 18

/* features [n_elems][18] (FP32) and "the limiter looks at this cell" flags [n_elems] of the current
 * state, in ascending element-ID order, into caller-owned device buffers (d_ok may be NULL) */
int32_t dgsw_rkdg_indicator_features(dgsw_handle h, float* d_features, uint8_t* d_ok);
/* one RK stage (as dgsw_rkdg_stage) with the plain limiter, recording the features of the state the
 * limiter sees and its decisions as labels: 1 changed, 0 unchanged, 255 not looked at (device buffers,
 * ascending element-ID order) - the training data of the indicator */
int32_t dgsw_rkdg_stage_record(dgsw_handle h, float* d_features, uint8_t* d_labels);
/* mode 0: plain limiter on every cell. mode 1: the MLP runs before each limiter pass and the limiter
 * visits only cells with p >= 1 - confidence (cells the network is not confident are smooth fall back to
 * the plain limiter). mode 2 (evaluation): the plain limiter decides every cell but writes back only
 * the cells mode 1 would visit, counting the misses. params: host FP32 array of DGSW_MLP_NPARAM. */
int32_t dgsw_rkdg_set_indicator(dgsw_handle h, const float* params, double confidence, int32_t mode);
/* the 18 features the indicator reads (dgsw_rkdg_indicator_features, dgsw_rkdg_stage_record and the gate):
 * 0 (default) the scale-free characteristic set (fields in characteristic units, one common scale, TVB
 * ratio, Froude numbers); 1 the raw set: the p = 1 modal coefficients of ze, qx, qy and the three
 * neighbour cell means of each field (a network for it takes its input normalisation in its first layer) */
int32_t dgsw_rkdg_set_indicator_features(dgsw_handle h, int32_t feature_set);
/* accumulated counts since the last reset: [0] cells the limiter would look at, [1] cells sent to it,
 * [2] cells it changed, [3] cells it would have changed but the indicator skipped (mode 2) */
int32_t dgsw_rkdg_indicator_stats(dgsw_handle h, int64_t* counts, int32_t reset);

/* handle-free MLP kernels on caller-owned device buffers, stream-ordered on `stream` (NULL = default).
 * forward: p[n] = MLP(x[n][18]); tensor_cores = 1 for the BF16 tcgen05 path (synchronises the stream),
 * 0 for the FP32 CUDA-core path. grad: mean weighted binary cross-entropy
 * -[w y log p + (1 - y) log(1 - p)] over the batch (y in {0, 1}) and its gradient into d_grad
 * [DGSW_MLP_NPARAM]; d_loss (device, one double) may be NULL; d_work holds dgsw_mlp_grad_work_floats(n)
 * floats. The sums run in a fixed order: repeated calls give identical results. adam: one Adam step
 * (bias-corrected, step >= 1) on d_params with moment buffers d_m, d_v. */
int32_t dgsw_mlp_forward(const float* d_x, int64_t n, const float* d_params, float* d_p, int32_t tensor_cores,
                         void* stream);
int64_t dgsw_mlp_grad_work_floats(int64_t n);
int32_t dgsw_mlp_grad(const float* d_x, const uint8_t* d_y, int64_t n, const float* d_params, float pos_weight,
                      float* d_grad, float* d_work, int64_t work_floats, double* d_loss, void* stream);
int32_t dgsw_mlp_adam(float* d_params, float* d_m, float* d_v, const float* d_grad, int32_t step, float lr,
                      float beta1, float beta2, float eps, void* stream);

/* ---- kernel self-checks: the stage kernel's device functions on caller data ----------------------
 * Host arrays in and out (device scratch is allocated per call); no handle. They run the same device
 * code the stage kernel inlines, so known-answer vectors can be checked against the CUDA path itself.
 * precision: DGSW_FP64 or DGSW_FP32 (inputs are rounded to FP32 and the flux evaluated in FP32). */
/* LLF_flux (rkdg_swe_LLF_flux.hpp:7-60) as test/test_llf_flux.cpp calls it: q_in, q_ex [n][3], bath and
 * the spherical factor sp [n] (applied to the in side), unit normal [n][2] -> F [n][3] */
int32_t dgsw_check_llf_flux(int32_t precision, int64_t n, double g, const double* q_in, const double* q_ex,
                            const double* bath, const double* sp, const double* normal, double* F);
/* ISP::Internal::ComputeFlux at one Gauss point (rkdg_swe_is_internal.hpp:26-95): LLF, F_ex = -F_in, and
 * the wet/dry fix-ups for a dry side (wet flags [n] of each side, bathymetry of each side) */
int32_t dgsw_check_internal_flux(int32_t precision, int64_t n, double g, const double* q_in, const double* q_ex,
                                 const double* bath_in, const double* bath_ex, const double* sp, const double* normal,
                                 const uint8_t* wet_in, const uint8_t* wet_ex, double* F_in, double* F_ex);
/* wetting_drying_kernel (swe_post_wet_dry.hpp:6-145) on p = 1 elements as test/test_wetting_drying.cpp
 * drives it: modal q [n][3 var][3 dof], bathymetry at the vertices [n][3], h_o (threshold
 * 1e6 h_o eps as swe_pre_init_prob_params.hpp:36), wet flags in -> q_out, wet_out, went_dry (may be NULL) */
int32_t dgsw_check_wetting_drying(int64_t n, const double* q, const double* bath_vrtx, double h_o,
                                  const uint8_t* wet_in, double* q_out, uint8_t* wet_out, uint8_t* went_dry);

/* execution control */
int32_t dgsw_rkdg_set_stream(dgsw_handle h, void* cuda_stream);
int32_t dgsw_rkdg_synchronize(dgsw_handle h);
/* device time of the most recent dgsw_rkdg_step call's stage kernels, from CUDA events recorded on the
 * handle's stream around it: total milliseconds and number of stage-kernel launches */
int32_t dgsw_rkdg_last_step_timing(dgsw_handle h, double* ms, int64_t* kernel_launches);
/* dgsw_rkdg_step(h, nsteps) with the stages launched one by one (no step graph) and a CUDA event pair
 * recorded on the handle's stream around every stage-kernel launch (with its levee pass on meshes with
 * levees): the summed device time of those launches and their number (a measurement aid; the same
 * states result as from dgsw_rkdg_step) */
int32_t dgsw_rkdg_step_timed(dgsw_handle h, int32_t nsteps, double* stage_ms, int64_t* stage_launches);

#ifdef __cplusplus
}
#endif

#endif /* DGSW_RKDG_H */
