// C ABI of the RKDG library: handle lifecycle, uploads, the stage/step driver and reductions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/dgsw_rkdg.h"
#include "host_setup.h"
#include "indicator.cuh"
#include "limiter_kernel.cuh"
#include "quadrature.h"
#include "reduce_kernels.cuh"
#include "stage_kernel.cuh"
#include "trouble.cuh"
#include "levee.cuh"
#include "postprocess.cuh"

using namespace dgsw;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return fail(DGSW_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        n = count;
        return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

int make_l2_rule(L2Rule& R, std::string& err) {
    Rule2D r = triangle_rule(20);
    if ((int)r.w.size() != L2_NPT) {
        err = "unexpected L2 rule size";
        return DGSW_ERR_UNSUPPORTED;
    }
    std::memset(&R, 0, sizeof(R));
    for (int i = 0; i < L2_NPT; ++i) {
        R.w[i] = r.w[i];
        R.psi[0][i] = -(r.z1[i] + r.z2[i]) / 2;
        R.psi[1][i] = (1 + r.z1[i]) / 2;
        R.psi[2][i] = (1 + r.z2[i]) / 2;
    }
    eval_basis(1, r.z1.data(), r.z2.data(), L2_NPT, R.phi[0]);
    eval_basis(2, r.z1.data(), r.z2.data(), L2_NPT, R.phi[1]);
    return DGSW_OK;
}

__global__ void advance_clock_kernel(DevClock* c, double dt) {
    c->t += dt;  // ESSPRKStepper::operator++ (explicit_ssp_rk_stepper.hpp:55-58)
    c->step += 1;
}

}  // namespace

namespace dgsw {
// the per-thread error message for entry points defined in other translation units
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace dgsw

struct dgsw_rkdg_s {
    dgsw_config cfg;
    Tables tb;
    Topology topo;
    Tiling tiling;
    dgsw_rk_table rk;
    int device = 0;
    int ns = 0, nd = 0;
    int64_t ne = 0, ne_pad = 0, nn = 0;
    bool fp32 = false;
    double h_o_thr = 1.0e-6;
    std::vector<double> node_xyz;
    std::vector<bool> need_sol;  // sol_k kept for later stages
    // device buffers
    size_t real_size = 8;
    std::vector<void*> Q;    // ns+1 stage states
    std::vector<void*> SOL;  // stored stage solutions (only where needed)
    // stage increments (FP32 precision without wetting/drying, limiter or levees, unless fp64_stages): the
    // carried state lives as two FP32 parts QF[qswap] + QL[qswap] (leading and trailing), the intermediate
    // stage states as FP32 increments D[s] = q_s - q_0 (s = 1 .. ns-1); the FP64 arrays Q[s] are formed only
    // when the host API reads a state, and split again after it writes one
    bool split = false;
    void* QF[2] = {nullptr, nullptr};  // the carried state's leading FP32 part (ping-pong pair)
    void* QL[2] = {nullptr, nullptr};  // and its trailing part
    std::vector<void*> D;     // [ns], D[0] unused
    std::vector<void*> DSOL;  // FP32 stored stage solutions (only where needed)
    void* bath = nullptr;  // [3][ne_pad] bathymetry modes of the linear part
    void* geo = nullptr;   // [5][ne_pad] J^-1 and |J|
    void* egeo = nullptr;  // [3][n_edges] edge normal and half length
    void* manning = nullptr;  // [ne_pad] g n^2 per element (Manning friction only)
    Forcing forcing;
    DBuf<int2> fface;      // tide / flow forcing records
    DBuf<double> fcon;
    int64_t n_levee = 0;   // levee interfaces
    DBuf<int4> lev;        // in element, in face, ex element, ex face (device order)
    DBuf<double> ldat;     // normal, crest height and coefficients at the Gauss points, spherical factors
    DBuf<double> levF;     // this stage's levee fluxes
    DBuf<unsigned char> went_dry;  // wet_dry_state.went_completely_dry (wetting/drying only)
    DBuf<double> post;             // output values for the writers (allocated on first use)
    DBuf<unsigned char> post_flags;
    DBuf<int2> halo;
    DBuf<int> tile_halo_off;
    DBuf<int> enodes, tile_edge_off, ref_of_dev;
    DBuf<int2> eslot;
    DBuf<int4> edges;
    DBuf<double2> xy;
    DBuf<double> nz;
    DBuf<unsigned char> wet[2];
    int wet_cur = 0;
    DBuf<DevStatus> status;
    DBuf<DevClock> clock;
    DBuf<double> red;  // reduction partials
    DBuf<unsigned char> limited;
    DBuf<int> nbr;     // neighbours per face, device order (limiter)
    DBuf<double> baryctr;  // barycentre values of the newest state (limiter)
    DBuf<double> lgeo;     // limiter geometry per element, [16][ne_pad]
    DBuf<float> lgeo_f;    // its first 15 rows in FP32 (the FP32 limiter form)
    // trouble indicator (computed in each limiter pass only when asked for)
    int trouble_on = 0;
    DBuf<signed char> nbr_face;  // [3][ne_pad] the neighbour's face across each face
    DBuf<double> tI;
    DBuf<unsigned char> tflag, tscratch, tout;
    int64_t device_bytes = 0;
    // stepper mirror on the host (ESSPRKStepper state)
    double t = 0.0;
    int64_t step = 0;
    int stage = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    // graphs of GRAPH_MULTI consecutive steps, same keys (for batches of many steps: one graph launch, and
    // no gap between graphs, per GRAPH_MULTI steps; small meshes are launch-bound)
    cudaGraphExec_t graph_multi[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t graph_multi_launches[4] = {0, 0, 0, 0};
    int qswap = 0;  // parity of the q_0 <-> q_ns swaps so far
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // per-launch timing of the stage kernel (dgsw_rkdg_step_timed): event pairs, recorded while kt_on
    std::vector<cudaEvent_t> kt_ev;
    bool kt_on = false;
    size_t kt_used = 0;
    DBuf<L2Rule> l2rule;
    DBuf<double> staging;  // FP64 host-layout state for the host API (allocated on first use)
    double last_ms = 0.0;
    int64_t last_launches = 0;
    size_t smem_bytes = 0;
    int tile = 256;
    int64_t graph_launches[4] = {0, 0, 0, 0};  // kernels one replay of graph[key] launches
    // ensemble members: element ranges [member_first[m], member_first[m+1]) in reference order
    int32_t n_members = 1;
    std::vector<int64_t> member_first;
    // autotuner record: candidate tile sizes and their measured device time per step
    int32_t n_tuned = 0;
    int32_t tuned_tile[DGSW_TUNE_MAX_CANDIDATES] = {0};
    int32_t tuned_occ[DGSW_TUNE_MAX_CANDIDATES] = {0};
    int32_t tuned_order[DGSW_TUNE_MAX_CANDIDATES] = {0};
    double tuned_ms[DGSW_TUNE_MAX_CANDIDATES] = {0};
    // stage-kernel register budget (0 default, 1 the alternative) and tile order (0 alternating, 1 ascending)
    int occ = 0, order = 0;
    int uncapped = 0;  // 1: the stage kernel with run-time shared-memory strides even where the caps fit
    // troubled-cell indicator (mode 0 off, 1 gate the limiter, 2 shadow: plain limiter, misses counted)
    int ind_mode = 0;
    int ind_fset = 0;  // indicator feature set (IND_FEATURES_*)
    float ind_skip_below = 0.1f;
    DBuf<float> ind_params;
    DBuf<int> ind_list;
    DBuf<int> ind_count;
    DBuf<unsigned char> ind_gate;
    DBuf<unsigned long long> ind_counters;
    DBuf<int> ind_error;
    int sm_count = 148;
};

namespace {

// steps per multi-step graph
constexpr int GRAPH_MULTI = 8;

template <typename Real>
void fill_stage_args(dgsw_rkdg_s* h, int s, StageArgs<Real>& A) {
    std::memset(&A, 0, sizeof(A));
    int n = 0;
    for (int k = 0; k < s; ++k) {
        if (h->rk.ark[s][k] != 0.0 || h->rk.brk[s][k] != 0.0) {
            A.qk[n] = (const double*)h->Q[k];
            A.solk[n] = (const double*)h->SOL[k];
            A.a[n] = h->rk.ark[s][k];
            A.bdt[n] = h->cfg.dt * h->rk.brk[s][k];
            ++n;
        }
    }
    A.qk[n] = (const double*)h->Q[s];
    A.solk[n] = nullptr;
    A.a[n] = h->rk.ark[s][s];
    A.bdt[n] = h->cfg.dt * h->rk.brk[s][s];
    ++n;
    A.nterms = n;
    A.store_sol = h->need_sol[s] ? 1 : 0;
    A.sol_out = (double*)h->SOL[s];
    A.q_out = (double*)h->Q[s + 1];
    if (h->split) {
        // the same terms as increments: q_0's term has none (d_0 = 0), q_k's is D[k]
        int m = 0;
        for (int k = 0; k < s; ++k)
            if (h->rk.ark[s][k] != 0.0 || h->rk.brk[s][k] != 0.0) {
                A.dk[m] = k ? (const Real*)h->D[k] : nullptr;
                A.dsolk[m] = (const Real*)h->DSOL[k];
                ++m;
            }
        A.dk[m] = s ? (const Real*)h->D[s] : nullptr;
        A.dsolk[m] = nullptr;
        A.q0f = (const Real*)h->QF[h->qswap];
        A.q0lo = (const Real*)h->QL[h->qswap];
        A.last = s + 1 == h->ns ? 1 : 0;
        A.d_out = A.last ? nullptr : (Real*)h->D[s + 1];
        A.q0f_out = A.last ? (Real*)h->QF[1 - h->qswap] : nullptr;
        A.q0lo_out = A.last ? (Real*)h->QL[1 - h->qswap] : nullptr;
        A.dsol_out = (Real*)h->DSOL[s];
    }
    A.bath = (const Real*)h->bath;
    A.geo = (const Real*)h->geo;
    A.enodes = h->enodes.p;
    A.eslot = h->eslot.p;
    A.edges = h->edges.p;
    A.egeo = (const Real*)h->egeo;
    A.tile_edge_off = h->tile_edge_off.p;
    A.halo = h->halo.p;
    A.tile_halo_off = h->tile_halo_off.p;
    A.n_edges = (int)(h->tiling.edges.size() / 4);
    A.xy = h->xy.p;
    A.nz = h->nz.p;
    A.ref_of_dev = h->ref_of_dev.p;
    A.baryctr = h->cfg.slope_limiting ? h->baryctr.p : nullptr;
    A.status = h->status.p;
    A.clock = h->clock.p;
    A.drk_s = h->cfg.dt * h->rk.drk[s];
    A.stage_index = s;
    A.nstages = h->ns;
    A.ne = (int)h->ne;
    A.ne_pad = (int)h->ne_pad;
    A.g = h->cfg.g;
    A.h_o = h->cfg.h_o;
    A.h_o_thr = h->h_o_thr;
    A.fn_set = h->cfg.function_set;
    for (int i = 0; i < 16; ++i) A.fn_params[i] = h->cfg.fn_params[i];
    A.spherical = h->cfg.spherical;
    A.sp_cos_lat0 = std::cos(h->cfg.sp_lat0_deg * 3.14159265359 / 180.0);  // the reference's PI
    A.sp_R = h->cfg.sp_R;
    A.friction = h->cfg.bottom_friction;
    A.friction_cf = h->cfg.friction_cf;
    A.manning = (const Real*)h->manning;
    A.fface = h->fface.p;
    A.fcon = h->fcon.p;
    // ESSPRKStepper keeps ramp = 1 when Utilities::almost_equal(ramp_duration, 0)
    A.ramp_on = std::fabs(h->cfg.ramp_duration) < std::numeric_limits<double>::epsilon() * 100 ? 0 : 1;
    A.ramp_duration = h->cfg.ramp_duration;
    A.went_dry = h->went_dry.p;
    // tile order alternates from stage to stage, across steps too (qswap flips once per step and keys
    // the step graphs), so that each stage starts where the previous one ended
    A.reverse = h->order == 0 ? ((s + h->qswap * h->ns) & 1) : 0;
}

cudaError_t launch_stage_any(dgsw_rkdg_s* h, const StageArgs<double>& A, int mode) {
    const int nt = (int)h->tiling.ntiles, mh = h->tiling.max_halo, me = h->tiling.max_edges;
    if (h->uncapped) mode |= STAGE_MODE_UNCAPPED;
    if (h->occ)
        return h->cfg.p == 1 ? launch_stage_p1_f64_occ(A, h->tile, nt, mh, me, mode, h->stream)
                             : launch_stage_p2_f64_occ(A, h->tile, nt, mh, me, mode, h->stream);
    return h->cfg.p == 1 ? launch_stage_p1_f64(A, h->tile, nt, mh, me, mode, h->stream)
                         : launch_stage_p2_f64(A, h->tile, nt, mh, me, mode, h->stream);
}
cudaError_t launch_stage_any(dgsw_rkdg_s* h, const StageArgs<float>& A, int mode) {
    const int nt = (int)h->tiling.ntiles, mh = h->tiling.max_halo, me = h->tiling.max_edges;
    if (h->uncapped) mode |= STAGE_MODE_UNCAPPED;
    if (h->split) {
        const int m = mode | (h->occ ? STAGE_MODE_OCC : 0);
        return h->cfg.p == 1 ? launch_stage_p1_f32_split(A, h->tile, nt, mh, me, m, h->stream)
                             : launch_stage_p2_f32_split(A, h->tile, nt, mh, me, m, h->stream);
    }
    if (h->occ)
        return h->cfg.p == 1 ? launch_stage_p1_f32_occ(A, h->tile, nt, mh, me, mode, h->stream)
                             : launch_stage_p2_f32_occ(A, h->tile, nt, mh, me, mode, h->stream);
    return h->cfg.p == 1 ? launch_stage_p1_f32(A, h->tile, nt, mh, me, mode, h->stream)
                         : launch_stage_p2_f32(A, h->tile, nt, mh, me, mode, h->stream);
}

template <typename Real>
cudaError_t launch_stage(dgsw_rkdg_s* h, int s) {
    StageArgs<Real> A;
    fill_stage_args<Real>(h, s, A);
    A.wet_in = h->wet[h->wet_cur].p;
    A.wet_out = h->wet[1 - h->wet_cur].p;
    if (h->n_levee) {
        // the levee interfaces' fluxes of this stage, ahead of the stage kernel that lifts them
        LeveeArgs<Real> L;
        L.q = (const double*)h->Q[s];
        L.bath = (const Real*)h->bath;
        L.wet = A.wet_in;
        L.lev = h->lev.p;
        L.ldat = h->ldat.p;
        L.F = h->levF.p;
        L.n = (int)h->n_levee;
        L.ne_pad = (int)h->ne_pad;
        L.g = h->cfg.g;
        cudaError_t e = launch_levee<Real>(L, h->cfg.p, h->stream);
        if (e != cudaSuccess) return e;
        A.levF = h->levF.p;
    }
    const int mode = (h->cfg.wetting_drying ? 1 : 0) | (h->cfg.function_source ? 2 : 0) |
                     (h->cfg.bottom_friction != DGSW_FRICTION_NONE ? 4 : 0);
    return launch_stage_any(h, A, mode);
}

template <typename Real>
cudaError_t launch_limiter(dgsw_rkdg_s* h, int s_out) {
    LimiterArgs<Real> L;
    std::memset(&L, 0, sizeof(L));
    L.q = (Real*)h->Q[s_out];
    L.baryctr = h->baryctr.p;
    L.wet = h->wet[h->wet_cur].p;
    L.nbr = h->nbr.p;
    L.enodes = h->enodes.p;
    L.xy = h->xy.p;
    L.nz = h->nz.p;
    L.limited = h->limited.p;
    L.ne = (int)h->ne;
    L.ne_pad = (int)h->ne_pad;
    L.g = h->cfg.g;
    L.M = h->cfg.sl_M;
    L.nu = h->cfg.sl_nu;
    L.status = h->status.p;
    L.ref_of_dev = h->ref_of_dev.p;
    L.lgeo = h->lgeo.p;
    L.lgeo_f = h->lgeo_f.p;
    // the FP32 path limits in FP32 arithmetic (FP64 differences, decisions free of rounding noise)
    const bool f32 = h->fp32 && !h->cfg.fp64_limiter;
    if (h->ind_mode == 1) {
        L.list = h->ind_list.p;
        L.list_count = h->ind_count.p;
        L.counters = h->ind_counters.p;
        return launch_limiter_kernel<Real>(L, h->cfg.p, h->stream, 8 * h->sm_count, f32);
    }
    if (h->ind_mode == 2) {
        L.gate = h->ind_gate.p;
        L.counters = h->ind_counters.p;
    }
    return launch_limiter_kernel<Real>(L, h->cfg.p, h->stream, 0, f32);
}

template <typename Real>
FeatureArgs<Real> feature_args(dgsw_rkdg_s* h, int s_out) {
    FeatureArgs<Real> F;
    F.q = (const Real*)h->Q[s_out];
    F.wet = h->wet[h->wet_cur].p;
    F.nbr = h->nbr.p;
    F.enodes = h->enodes.p;
    F.xy = h->xy.p;
    F.nz = h->nz.p;
    F.ne = (int)h->ne;
    F.ne_pad = (int)h->ne_pad;
    F.nd = h->nd;
    F.g = h->cfg.g;
    F.M = h->cfg.sl_M;
    F.fset = h->ind_fset;
    return F;
}

// the indicator pass before the limiter: features + MLP on the tensor cores -> work list or gate flags
template <typename Real>
cudaError_t launch_indicator_gate(dgsw_rkdg_s* h, int s_out) {
    TcArgs T;
    std::memset(&T, 0, sizeof(T));
    T.params = h->ind_params.p;
    T.mode = h->ind_mode;
    T.skip_below = h->ind_skip_below;
    T.list = h->ind_list.p;
    T.list_count = h->ind_count.p;
    T.gate = h->ind_gate.p;
    T.limited = h->limited.p;
    T.counters = h->ind_counters.p;
    T.error = h->ind_error.p;
    if (h->ind_mode == 1) {
        cudaError_t e = cudaMemsetAsync(h->ind_count.p, 0, sizeof(int), h->stream);
        if (e != cudaSuccess) return e;
    }
    return launch_mlp_tc<Real>(T, feature_args<Real>(h, s_out), h->stream);
}

struct StageRecord {
    float* features;  // [ne][18], reference order (device)
    uint8_t* labels;  // [ne], reference order (device): limiter decision, 255 where it does not look
};

__global__ void record_labels_kernel(const unsigned char* limited, const int* ref_of_dev, int ne, uint8_t* labels) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ne) return;
    const int r = ref_of_dev[d];
    labels[r] = labels[r] ? limited[d] : (uint8_t)255;
}

cudaError_t split_form(dgsw_rkdg_s* h, int s);

// one RK stage: stage kernel, (clock on the last stage), indicator, limiter, wet flag buffer flip
cudaError_t enqueue_stage(dgsw_rkdg_s* h, int s, int64_t& launches, const StageRecord* rec = nullptr) {
    const bool timed = h->kt_on && h->kt_used + 2 <= h->kt_ev.size();
    if (timed) {
        cudaError_t e = cudaEventRecord(h->kt_ev[h->kt_used], h->stream);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = h->fp32 ? launch_stage<float>(h, s) : launch_stage<double>(h, s);
    if (e != cudaSuccess) return e;
    if (timed) {
        e = cudaEventRecord(h->kt_ev[h->kt_used + 1], h->stream);
        if (e != cudaSuccess) return e;
        h->kt_used += 2;
    }
    launches += h->n_levee ? 2 : 1;
    h->wet_cur = 1 - h->wet_cur;
    int s_out = s + 1;
    if (s + 1 == h->ns) {
        advance_clock_kernel<<<1, 1, 0, h->stream>>>(h->clock.p, h->cfg.dt);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ++launches;
        std::swap(h->Q[0], h->Q[h->ns]);  // UpdateState's swap of q_0 and q_ns
        h->qswap ^= 1;
        s_out = 0;
    }
    if (rec) {
        // features of the state the limiter is about to see; ok flags into the label buffer
        e = split_form(h, s_out);
        if (e != cudaSuccess) return e;
        e = launch_indicator_features<double>(feature_args<double>(h, s_out), h->ref_of_dev.p, rec->features,
                                              rec->labels, h->stream);
        if (e != cudaSuccess) return e;
        ++launches;
    }
    if (h->cfg.slope_limiting && h->trouble_on) {
        TroubleArgs<double> T;
        TroubleArgs<float> Tf;
        auto fill = [&](auto& X, auto bath) {
            std::memset(&X, 0, sizeof(X));
            X.q = (const double*)h->Q[s_out];
            X.bath = bath;
            X.wet = h->wet[h->wet_cur].p;
            X.nbr = h->nbr.p;
            X.nbr_face = h->nbr_face.p;
            X.enodes = h->enodes.p;
            X.xy = h->xy.p;
            X.ref_of_dev = h->ref_of_dev.p;
            X.I = h->tI.p;
            X.flag = h->tflag.p;
            X.ne = (int)h->ne;
            X.ne_pad = (int)h->ne_pad;
        };
        if (h->fp32) {
            fill(Tf, (const float*)h->bath);
            e = launch_trouble<float>(Tf, h->cfg.p, h->tscratch.p, h->tout.p, h->stream);
        } else {
            fill(T, (const double*)h->bath);
            e = launch_trouble<double>(T, h->cfg.p, h->tscratch.p, h->tout.p, h->stream);
        }
        if (e != cudaSuccess) return e;
        launches += 6;
    }
    if (h->cfg.slope_limiting) {
        const int mode = h->ind_mode;
        if (rec) h->ind_mode = 0;  // labels come from the plain limiter
        if (h->ind_mode) {
            e = launch_indicator_gate<double>(h, s_out);
            if (e != cudaSuccess) return e;
            ++launches;
        }
        e = launch_limiter<double>(h, s_out);
        h->ind_mode = mode;
        if (e != cudaSuccess) return e;
        ++launches;
    }
    if (rec) {
        if (!h->cfg.slope_limiting) {
            e = cudaMemsetAsync(h->limited.p, 0, h->ne_pad, h->stream);
            if (e != cudaSuccess) return e;
        }
        record_labels_kernel<<<(unsigned)((h->ne + 255) / 256), 256, 0, h->stream>>>(h->limited.p, h->ref_of_dev.p,
                                                                                     (int)h->ne, rec->labels);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ++launches;
    }
    return cudaSuccess;
}

void advance_host_stepper(dgsw_rkdg_s* h) {
    h->stage = (h->stage + 1) % h->ns;
    if (h->stage == 0) {
        h->t += h->cfg.dt;
        h->step += 1;
    }
}

int check_status(dgsw_rkdg_s* h) {
    DevStatus st;
    CUDA_TRY(cudaMemcpyAsync(&st, h->status.p, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (st.nan_flag) {
        // the first stage with a NaN and its smallest element, as the reference's per-stage scrutiny
        // reports it before aborting
        const uint32_t ref = (uint32_t)(st.nan_key & 0xffffffffull);
        const unsigned long long counter = st.nan_key >> 32;
        uint32_t id = ref < h->topo.ids.size() ? h->topo.ids[ref] : 0;
        DevStatus z;
        std::memset(&z, 0, sizeof(z));
        z.nan_key = ~0ull;
        cudaMemcpyAsync(h->status.p, &z, sizeof(z), cudaMemcpyHostToDevice, h->stream);
        cudaStreamSynchronize(h->stream);
        return fail(DGSW_ERR_NAN, "Fatal Error: NaN found at element " + std::to_string(id) + " (step " +
                                      std::to_string(counter / (unsigned long long)h->ns) + ", stage " +
                                      std::to_string(counter % (unsigned long long)h->ns) + ")");
    }
    return DGSW_OK;
}

void destroy_graphs(dgsw_rkdg_s* h) {
    for (int i = 0; i < 4; ++i) {
        if (h->graph[i]) {
            cudaGraphExecDestroy(h->graph[i]);
            h->graph[i] = nullptr;
        }
        if (h->graph_multi[i]) {
            cudaGraphExecDestroy(h->graph_multi[i]);
            h->graph_multi[i] = nullptr;
        }
    }
}

int ensure_staging(dgsw_rkdg_s* h) {
    if (h->staging.p) return DGSW_OK;
    cudaError_t e = h->staging.alloc((size_t)h->ne * 3 * h->nd);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("staging alloc: ") + cudaGetErrorString(e));
    h->device_bytes += (int64_t)h->ne * 3 * h->nd * 8;
    return DGSW_OK;
}

// Stage increments and the FP64 stage states, for the host API's reads and writes: a state written
// through the API is turned into what the increment kernels read (the carried state's two FP32 parts at
// stage 0, the increment D[s] from q_0 after it), and a state read through the API is formed from them
// (Q[s] = q0f + q0lo + D[s], FP64; q0f + q0lo is exact in FP64)
__global__ void split_carry_kernel(const double* __restrict__ q, float* __restrict__ hi, float* __restrict__ lo,
                                   size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float h = (float)q[i];
        hi[i] = h;
        lo[i] = (float)(q[i] - (double)h);
    }
}

__global__ void split_incr_kernel(const double* __restrict__ q, const float* __restrict__ hi,
                                  const float* __restrict__ lo, float* __restrict__ d, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = (float)(q[i] - ((double)hi[i] + (double)lo[i]));
}

__global__ void split_form_kernel(const float* __restrict__ hi, const float* __restrict__ lo,
                                  const float* __restrict__ d, double* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double q0 = (double)hi[i] + (double)lo[i];
        out[i] = d ? q0 + (double)d[i] : q0;
    }
}

unsigned split_grid(dgsw_rkdg_s* h, size_t n) {
    return (unsigned)std::min<size_t>((n + 255) / 256, (size_t)8 * h->sm_count);
}

// after Q[h->stage] was written through the API
cudaError_t split_absorb(dgsw_rkdg_s* h) {
    if (!h->split) return cudaSuccess;
    const size_t n = (size_t)3 * h->nd * h->ne_pad;
    float* hi = (float*)h->QF[h->qswap];
    float* lo = (float*)h->QL[h->qswap];
    if (h->stage == 0)
        split_carry_kernel<<<split_grid(h, n), 256, 0, h->stream>>>((const double*)h->Q[0], hi, lo, n);
    else
        split_incr_kernel<<<split_grid(h, n), 256, 0, h->stream>>>((const double*)h->Q[h->stage], hi, lo,
                                                                   (float*)h->D[h->stage], n);
    return cudaGetLastError();
}

// before Q[s] is read outside the stage kernels
cudaError_t split_form(dgsw_rkdg_s* h, int s) {
    if (!h->split) return cudaSuccess;
    const size_t n = (size_t)3 * h->nd * h->ne_pad;
    split_form_kernel<<<split_grid(h, n), 256, 0, h->stream>>>((const float*)h->QF[h->qswap],
                                                               (const float*)h->QL[h->qswap],
                                                               s ? (const float*)h->D[s] : nullptr,
                                                               (double*)h->Q[s], n);
    return cudaGetLastError();
}

// host FP64 [ref][var][dof] -> one DMA into the staging buffer -> device permute + convert
int upload_state(dgsw_rkdg_s* h, const double* q) {
    int rc = ensure_staging(h);
    if (rc) return rc;
    const size_t bytes = (size_t)h->ne * 3 * h->nd * sizeof(double);
    CUDA_TRY(cudaMemcpyAsync(h->staging.p, q, bytes, cudaMemcpyHostToDevice, h->stream));
    cudaError_t e = launch_permute_in<double, double>(h->staging.p, (double*)h->Q[h->stage], h->ref_of_dev.p,
                                                      (int)h->ne, (int)h->ne_pad, 3 * h->nd, h->stream);
    if (e == cudaSuccess) e = split_absorb(h);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("set_state: ") + cudaGetErrorString(e));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

int download_state(dgsw_rkdg_s* h, double* q) {
    int rc = ensure_staging(h);
    if (rc) return rc;
    cudaError_t e = split_form(h, h->stage);
    if (e == cudaSuccess)
        e = launch_permute_out<double, double>((const double*)h->Q[h->stage], h->staging.p, h->ref_of_dev.p,
                                               (int)h->ne, (int)h->ne_pad, 3 * h->nd, h->stream);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("get_state: ") + cudaGetErrorString(e));
    const size_t bytes = (size_t)h->ne * 3 * h->nd * sizeof(double);
    CUDA_TRY(cudaMemcpyAsync(q, h->staging.p, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

int upload_wet(dgsw_rkdg_s* h, const uint8_t* wet_ref) {
    std::vector<unsigned char> w(h->ne_pad, 0);
    for (int64_t d = 0; d < h->ne; ++d) w[d] = wet_ref[h->tiling.ref_of_dev[d]] ? 1 : 0;
    CUDA_TRY(cudaMemcpyAsync(h->wet[h->wet_cur].p, w.data(), h->ne_pad, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

template <typename Real>
int run_reduction(dgsw_rkdg_s* h, int what, double* out) {
    ReduceArgs<Real> R;
    std::memset(&R, 0, sizeof(R));
    {
        cudaError_t ef = split_form(h, what == 0 ? 0 : h->stage);
        if (ef != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("reduction: ") + cudaGetErrorString(ef));
    }
    // the L2 error reads state[0] (swe_post_comp_res_l2.hpp:12), the mass the current stage state
    R.q = (const double*)h->Q[what == 0 ? 0 : h->stage];
    R.bath = (const Real*)h->bath;
    R.enodes = h->enodes.p;
    R.xy = h->xy.p;
    R.ne = (int)h->ne;
    R.ne_pad = (int)h->ne_pad;
    R.t = h->t + h->cfg.dt * h->rk.drk[h->stage];
    R.fn_set = h->cfg.function_set;
    for (int i = 0; i < 16; ++i) R.fn_params[i] = h->cfg.fn_params[i];
    R.partial = h->red.p;
    R.rule = h->l2rule.p;
    R.npartial = (int)h->red.n;
    cudaError_t e = launch_reduction<Real>(R, h->cfg.p, what, h->stream);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("reduction: ") + cudaGetErrorString(e));
    std::vector<double> part(h->red.n);
    CUDA_TRY(cudaMemcpyAsync(part.data(), h->red.p, h->red.n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    double s = 0.0;
    for (double v : part) s += v;  // fixed order: deterministic
    *out = s;
    return DGSW_OK;
}

}  // namespace

extern "C" {

int32_t dgsw_abi_version(void) { return DGSW_ABI_VERSION; }

const char* dgsw_last_error(void) { return g_last_error.c_str(); }

const char* dgsw_status_string(int32_t s) {
    switch (s) {
        case DGSW_OK:
            return "ok";
        case DGSW_ERR_INVALID_ARGUMENT:
            return "invalid argument";
        case DGSW_ERR_MESH:
            return "mesh error";
        case DGSW_ERR_CUDA:
            return "CUDA error";
        case DGSW_ERR_NAN:
            return "NaN in solution";
        case DGSW_ERR_UNSUPPORTED:
            return "unsupported";
        case DGSW_ERR_NO_DEVICE:
            return "no CUDA device";
        case DGSW_ERR_IO:
            return "I/O error";
        default:
            return "unknown status";
    }
}

void dgsw_config_default(dgsw_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->p = 1;
    c->rk_nstages = 2;
    c->rk_order = 2;
    c->dt = 1.0;
    c->g = 9.81;
    c->h_o = 0.1;
    c->sl_M = 1.0e-8;
    c->sl_nu = 1.5;
    c->sp_R = 6378200.0;
    c->precision = DGSW_FP64;
    c->tile = 0;
    c->renumber = 1;
    c->use_graphs = 1;
}

// create for one mesh; caller_group (per caller element, may be NULL) and group_params describe the
// members of an ensemble
static int32_t create_impl(const dgsw_config* cfg, const dgsw_mesh* mesh, const int32_t* caller_group,
                           int32_t n_groups, const double* group_params, dgsw_handle* out) {
    if (!cfg || !mesh || !out) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(DGSW_ERR_NO_DEVICE, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(DGSW_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    if (!(cfg->dt > 0)) return fail(DGSW_ERR_INVALID_ARGUMENT, "dt must be positive");
    if (cfg->precision != DGSW_FP64 && cfg->precision != DGSW_FP32)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "precision must be DGSW_FP64 or DGSW_FP32");
    if (cfg->function_set < 0 || cfg->function_set >= DGSW_FN_COUNT)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "unknown function set");
    if (cfg->bottom_friction < DGSW_FRICTION_NONE || cfg->bottom_friction > DGSW_FRICTION_MANNING)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "unknown bottom friction type");
    if (cfg->bottom_friction != DGSW_FRICTION_NONE && cfg->friction_cf < 0.)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "Fatal Error: Chezy friction coefficient must be postive!");
    if (cfg->bottom_friction == DGSW_FRICTION_MANNING && !mesh->node_manning_n)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "Manning friction needs the mesh's node_manning_n");
    auto* h = new dgsw_rkdg_s();
    h->cfg = *cfg;
    h->device = cfg->device;
    std::string err;
    int rc = build_tables(cfg->p, h->tb, err);
    if (rc) {
        delete h;
        return fail(rc, err);
    }
    if (dgsw_rk_table_init(cfg->rk_nstages, cfg->rk_order, &h->rk) != 0) {
        delete h;
        return fail(DGSW_ERR_INVALID_ARGUMENT, "Fatal Error: invalid Runge-Kutta method entered!");
    }
    h->ns = cfg->rk_nstages;
    h->nd = h->tb.nd;
    rc = build_topology(mesh, h->topo, err);
    if (!rc) rc = build_forcing(mesh, h->topo, cfg->p, h->forcing, err);
    if (rc) {
        delete h;
        return fail(rc, err);
    }
    if (caller_group) {
        h->topo.group.resize(h->topo.ne);
        for (int64_t r = 0; r < h->topo.ne; ++r) h->topo.group[r] = caller_group[h->topo.src[r]];
        h->topo.group_params.assign(group_params, group_params + (size_t)n_groups * DGSW_FN_PARAMS);
        h->n_members = n_groups;
        h->member_first.assign(n_groups + 1, 0);
        for (int64_t r = 0; r < h->topo.ne; ++r) h->member_first[h->topo.group[r] + 1]++;
        for (int32_t m = 0; m < n_groups; ++m) h->member_first[m + 1] += h->member_first[m];
    }
    h->ne = h->topo.ne;
    h->nn = mesh->n_nodes;
    h->ne_pad = (h->ne + 31) / 32 * 32;
    if ((int64_t)3 * h->nd * h->ne_pad >= ((int64_t)1 << 31)) {
        delete h;
        return fail(DGSW_ERR_UNSUPPORTED, "mesh too large for 32-bit state indexing on one handle");
    }
    h->fp32 = cfg->precision == DGSW_FP32;
    h->real_size = h->fp32 ? sizeof(float) : sizeof(double);
    if (cfg->wetting_drying) h->h_o_thr = 1.0e6 * cfg->h_o * std::numeric_limits<double>::epsilon();
    h->node_xyz.assign(mesh->node_xyz, mesh->node_xyz + 3 * mesh->n_nodes);
    int tile = cfg->tile;
    if (tile == 0) tile = 128;  // measured faster than 256 at p = 1 and p = 2 in both precisions
    if (tile != 128 && tile != 256) {
        delete h;
        return fail(DGSW_ERR_INVALID_ARGUMENT, "tile must be 0 (automatic), 128 or 256");
    }
    h->tile = tile;
    if ((cfg->occupancy != 0 && cfg->occupancy != 1) || (cfg->tile_order != 0 && cfg->tile_order != 1)) {
        delete h;
        return fail(DGSW_ERR_INVALID_ARGUMENT, "occupancy and tile_order must be 0 or 1");
    }
    h->occ = cfg->occupancy;
    h->order = cfg->tile_order;
    rc = build_tiling(h->topo, h->node_xyz.data(), tile, cfg->renumber != 0, h->tiling, err);
    if (rc) {
        delete h;
        return fail(rc, err);
    }
    // which stage solutions are read by later stages (off-diagonal brk)
    h->need_sol.assign(h->ns, false);
    for (int i = 0; i < h->ns; ++i)
        for (int k = 0; k < i; ++k)
            if (h->rk.brk[i][k] != 0.0) h->need_sol[k] = true;

    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
        delete h;
        return fail(DGSW_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    auto cleanup_fail = [&](const std::string& what, cudaError_t ce) {
        dgsw_rkdg_destroy(h);
        return fail(DGSW_ERR_CUDA, what + ": " + cudaGetErrorString(ce));
    };
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cleanup_fail("stream", e);
    h->own_stream = true;
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    if (h->sm_count <= 0) h->sm_count = 148;
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    const size_t state_bytes = (size_t)3 * h->nd * h->ne_pad * sizeof(double);  // FP64 states in both precisions
    h->Q.assign(h->ns + 1, nullptr);
    h->SOL.assign(h->ns, nullptr);
    for (int s = 0; s <= h->ns; ++s) {
        if ((e = cudaMalloc(&h->Q[s], state_bytes)) != cudaSuccess) return cleanup_fail("state alloc", e);
        cudaMemset(h->Q[s], 0, state_bytes);
        h->device_bytes += state_bytes;
    }
    for (int s = 0; s < h->ns; ++s)
        if (h->need_sol[s]) {
            if ((e = cudaMalloc(&h->SOL[s], state_bytes)) != cudaSuccess) return cleanup_fail("sol alloc", e);
            h->device_bytes += state_bytes;
        }
    const size_t bath_bytes = (size_t)3 * h->ne_pad * h->real_size;
    if ((e = cudaMalloc(&h->bath, bath_bytes)) != cudaSuccess) return cleanup_fail("bath alloc", e);
    h->device_bytes += bath_bytes;
    const size_t geo_bytes = (size_t)5 * h->ne_pad * h->real_size;
    if ((e = cudaMalloc(&h->geo, geo_bytes)) != cudaSuccess) return cleanup_fail("geometry alloc", e);
    h->device_bytes += geo_bytes;
    const size_t n_edges = h->tiling.edges.size() / 4;
    const size_t egeo_bytes = (size_t)3 * std::max<size_t>(n_edges, 1) * h->real_size;
    if ((e = cudaMalloc(&h->egeo, egeo_bytes)) != cudaSuccess) return cleanup_fail("edge geometry alloc", e);
    h->device_bytes += egeo_bytes;
    // static mesh data in device order
    {
        std::vector<int> en((size_t)3 * h->ne_pad, 0);
        std::vector<double> bathm;
        project_bathymetry(h->topo, h->node_xyz.data(), h->tb, bathm);
        std::vector<double> bdev((size_t)3 * h->ne_pad, 0.0);
        std::vector<double> gdev((size_t)5 * h->ne_pad, 0.0);
        std::vector<int> nb((size_t)3 * h->ne_pad, -1);
#pragma omp parallel for schedule(static)
        for (int64_t d = 0; d < h->ne; ++d) {
            int64_t r = h->tiling.ref_of_dev[d];
            for (int v = 0; v < 3; ++v) {
                en[(size_t)v * h->ne_pad + d] = h->topo.enodes[3 * r + v];
                int32_t n = h->topo.nbr[3 * r + v];
                // limiter neighbours: device index, -2 - type for faces without a neighbour
                nb[(size_t)v * h->ne_pad + d] =
                    n >= 0 ? h->tiling.dev_of_ref[n] : -2 - (int)h->topo.btype[3 * r + v];
            }
            // the projected bathymetry is linear: modes above the third are rounding residue
            for (int k = 0; k < 3; ++k) bdev[(size_t)k * h->ne_pad + d] = bathm[r * h->nd + k];
            double gg[5];
            element_geometry(h->node_xyz.data(), &h->topo.enodes[3 * r], gg);
            for (int c = 0; c < 5; ++c) gdev[(size_t)c * h->ne_pad + d] = gg[c];
        }
        if ((e = h->enodes.alloc(en.size())) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->enodes.p, en.data(), en.size() * sizeof(int), cudaMemcpyHostToDevice);
        if ((e = h->nbr.alloc(nb.size())) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->nbr.p, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice);
        std::vector<double> edev((size_t)3 * std::max<size_t>(n_edges, 1), 0.0);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n_edges; ++i)
            for (int c = 0; c < 3; ++c) edev[c * n_edges + i] = h->tiling.egeo[3 * i + c];
        auto upload_real = [&](void* dst, const std::vector<double>& src) {
            if (h->fp32) {
                std::vector<float> f(src.size());
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < (int64_t)src.size(); ++i) f[i] = (float)src[i];
                cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
            } else {
                cudaMemcpy(dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice);
            }
        };
        upload_real(h->bath, bdev);
        upload_real(h->geo, gdev);
        upload_real(h->egeo, edev);
        if (cfg->bottom_friction == DGSW_FRICTION_MANNING) {
            std::vector<double> mf, mdev((size_t)h->ne_pad, 0.0);
            manning_factor(h->topo, mesh->node_manning_n, cfg->g, mf);
            for (int64_t d = 0; d < h->ne; ++d) mdev[d] = mf[h->tiling.ref_of_dev[d]];
            if ((e = cudaMalloc(&h->manning, (size_t)h->ne_pad * h->real_size)) != cudaSuccess)
                return cleanup_fail("alloc", e);
            upload_real(h->manning, mdev);
            h->device_bytes += (int64_t)h->ne_pad * h->real_size;
        }
        static_assert(LEVEE_STRIDE == LEVEE_STRIDE_DEV, "levee record layout");
        {
            std::vector<double> ld;
            std::string e2;
            const int lrc = build_levees(mesh, h->topo, cfg->p, h->node_xyz.data(), *cfg, ld, e2);
            if (lrc) {
                dgsw_rkdg_destroy(h);
                return fail(lrc, e2);
            }
            h->n_levee = (int64_t)h->topo.intf.size() / 4 - h->topo.n_intf_internal;
            if (h->n_levee) {
                std::vector<int4> lv(h->n_levee);
                for (int64_t l = 0; l < h->n_levee; ++l) {
                    const int32_t* I = &h->topo.intf[4 * (h->topo.n_intf_internal + l)];
                    lv[l] = make_int4(h->tiling.dev_of_ref[I[0]], I[2], h->tiling.dev_of_ref[I[1]], I[3]);
                }
                if ((e = h->lev.alloc(h->n_levee)) != cudaSuccess || (e = h->ldat.alloc(ld.size())) != cudaSuccess ||
                    (e = h->levF.alloc((size_t)h->n_levee * 6 * MAX_NG)) != cudaSuccess)
                    return cleanup_fail("alloc", e);
                cudaMemcpy(h->lev.p, lv.data(), lv.size() * sizeof(int4), cudaMemcpyHostToDevice);
                cudaMemcpy(h->ldat.p, ld.data(), ld.size() * sizeof(double), cudaMemcpyHostToDevice);
                cudaMemset(h->levF.p, 0, (size_t)h->n_levee * 6 * MAX_NG * sizeof(double));
                h->device_bytes += (int64_t)(lv.size() * 16 + ld.size() * 8 + h->n_levee * 6 * MAX_NG * 8);
            }
        }
        static_assert(FORCE_STRIDE == FORCE_STRIDE_DEV, "forcing record layout");
        const size_t nff = h->forcing.face.size() / 2, nfc = h->forcing.con.size();
        if (nff) {
            if ((e = h->fface.alloc(nff)) != cudaSuccess) return cleanup_fail("alloc", e);
            cudaMemcpy(h->fface.p, h->forcing.face.data(), nff * sizeof(int2), cudaMemcpyHostToDevice);
            if ((e = h->fcon.alloc(std::max<size_t>(nfc, 1))) != cudaSuccess) return cleanup_fail("alloc", e);
            if (nfc) cudaMemcpy(h->fcon.p, h->forcing.con.data(), nfc * sizeof(double), cudaMemcpyHostToDevice);
            h->device_bytes += (int64_t)(nff * 8 + nfc * 8);
        }
        const size_t nhalo = h->tiling.halo.size() / 2;
        if ((e = h->halo.alloc(std::max<size_t>(nhalo, 1))) != cudaSuccess) return cleanup_fail("alloc", e);
        if (nhalo) cudaMemcpy(h->halo.p, h->tiling.halo.data(), nhalo * sizeof(int2), cudaMemcpyHostToDevice);
        if ((e = h->tile_halo_off.alloc(h->tiling.tile_halo_off.size())) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->tile_halo_off.p, h->tiling.tile_halo_off.data(), h->tiling.tile_halo_off.size() * sizeof(int),
                   cudaMemcpyHostToDevice);
        std::vector<double2> xy(h->nn);
        std::vector<double> nz(h->nn);
        for (int64_t i = 0; i < h->nn; ++i) {
            xy[i] = make_double2(h->node_xyz[3 * i], h->node_xyz[3 * i + 1]);
            nz[i] = h->node_xyz[3 * i + 2];
        }
        if ((e = h->xy.alloc(h->nn)) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->xy.p, xy.data(), h->nn * sizeof(double2), cudaMemcpyHostToDevice);
        if ((e = h->nz.alloc(h->nn)) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->nz.p, nz.data(), h->nn * sizeof(double), cudaMemcpyHostToDevice);
        const size_t nedges = n_edges;
        if ((e = h->edges.alloc(std::max<size_t>(nedges, 1))) != cudaSuccess) return cleanup_fail("alloc", e);
        if (nedges) cudaMemcpy(h->edges.p, h->tiling.edges.data(), nedges * sizeof(int4), cudaMemcpyHostToDevice);
        if ((e = h->tile_edge_off.alloc(h->tiling.tile_edge_off.size())) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->tile_edge_off.p, h->tiling.tile_edge_off.data(), h->tiling.tile_edge_off.size() * sizeof(int),
                   cudaMemcpyHostToDevice);
        if ((e = h->eslot.alloc(h->ne)) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->eslot.p, h->tiling.eslot.data(), h->ne * sizeof(int2), cudaMemcpyHostToDevice);
        if ((e = h->ref_of_dev.alloc(h->ne)) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemcpy(h->ref_of_dev.p, h->tiling.ref_of_dev.data(), h->ne * sizeof(int), cudaMemcpyHostToDevice);
        for (int i = 0; i < 2; ++i) {
            if ((e = h->wet[i].alloc(h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
            cudaMemset(h->wet[i].p, 1, h->ne_pad);
        }
        if ((e = h->limited.alloc(h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
        if (cfg->slope_limiting) {
            if ((e = h->baryctr.alloc((size_t)3 * h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
            cudaMemset(h->baryctr.p, 0, (size_t)3 * h->ne_pad * sizeof(double));
            h->device_bytes += (int64_t)3 * h->ne_pad * 8;
        }
        cudaMemset(h->limited.p, 0, h->ne_pad);
        if (cfg->wetting_drying) {
            if ((e = h->went_dry.alloc(h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
            cudaMemset(h->went_dry.p, 0, h->ne_pad);
        }
        if ((e = h->status.alloc(1)) != cudaSuccess) return cleanup_fail("alloc", e);
        DevStatus z;
        std::memset(&z, 0, sizeof(z));
        z.nan_key = ~0ull;
        cudaMemcpy(h->status.p, &z, sizeof(z), cudaMemcpyHostToDevice);
        if ((e = h->clock.alloc(1)) != cudaSuccess) return cleanup_fail("alloc", e);
        cudaMemset(h->clock.p, 0, sizeof(DevClock));
        if ((e = h->red.alloc(reduction_partials(h->ne))) != cudaSuccess) return cleanup_fail("alloc", e);
        {
            static L2Rule Rh;
            std::string e2;
            if (make_l2_rule(Rh, e2) != DGSW_OK) {
                dgsw_rkdg_destroy(h);
                return fail(DGSW_ERR_UNSUPPORTED, e2);
            }
            if ((e = h->l2rule.alloc(1)) != cudaSuccess) return cleanup_fail("alloc", e);
            cudaMemcpy(h->l2rule.p, &Rh, sizeof(L2Rule), cudaMemcpyHostToDevice);
        }
        h->device_bytes += en.size() * 4 + nb.size() * 4 + h->nn * 24 + nedges * 16 + h->ne * 12 + 3 * h->ne_pad;
    }
    if (cfg->slope_limiting) {
        // the limiter's geometry, once (the same device code the limiter would run per stage)
        if ((e = h->lgeo.alloc((size_t)LIM_GEO * h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
        h->device_bytes += (int64_t)LIM_GEO * h->ne_pad * 8;
        LimiterArgs<double> L;
        std::memset(&L, 0, sizeof(L));
        L.nbr = h->nbr.p;
        L.enodes = h->enodes.p;
        L.xy = h->xy.p;
        L.nz = h->nz.p;
        L.ne = (int)h->ne;
        L.ne_pad = (int)h->ne_pad;
        if (h->fp32 && !cfg->fp64_limiter) {
            if ((e = h->lgeo_f.alloc((size_t)(LIM_GEO - 1) * h->ne_pad)) != cudaSuccess) return cleanup_fail("alloc", e);
            h->device_bytes += (int64_t)(LIM_GEO - 1) * h->ne_pad * 4;
        }
        limiter_geometry_kernel<double><<<(unsigned)((h->ne + 255) / 256), 256, 0, h->stream>>>(L, h->lgeo.p,
                                                                                                h->lgeo_f.p);
        if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cleanup_fail("limiter geometry", e);
    }
    // stage increments: FP32 arithmetic on a configuration whose stage states only the stage kernel reads
    // (no wetting/drying, slope limiter or levee pass, which work on the FP64 states), with at least three
    // stages (measured on 524,288 triangles: p = 2 SSP-RK3 1.6-2.5 % faster per step; p = 1 SSP-RK2, where
    // only one intermediate state exists, 2-3 % slower)
    h->split = h->fp32 && !cfg->fp64_stages && !cfg->wetting_drying && !cfg->slope_limiting && h->n_levee == 0 &&
               h->ns >= 3;
    if (h->split) {
        const size_t nval = (size_t)3 * h->nd * h->ne_pad;
        h->D.assign(h->ns, nullptr);
        h->DSOL.assign(h->ns, nullptr);
        for (int i = 0; i < 2; ++i) {
            if ((e = cudaMalloc(&h->QF[i], nval * sizeof(float))) != cudaSuccess) return cleanup_fail("state alloc", e);
            if ((e = cudaMalloc(&h->QL[i], nval * sizeof(float))) != cudaSuccess) return cleanup_fail("state alloc", e);
            cudaMemset(h->QF[i], 0, nval * sizeof(float));
            cudaMemset(h->QL[i], 0, nval * sizeof(float));
            h->device_bytes += 2 * nval * sizeof(float);
        }
        for (int s = 1; s < h->ns; ++s) {
            if ((e = cudaMalloc(&h->D[s], nval * sizeof(float))) != cudaSuccess) return cleanup_fail("state alloc", e);
            cudaMemset(h->D[s], 0, nval * sizeof(float));
            h->device_bytes += nval * sizeof(float);
        }
        for (int s = 0; s < h->ns; ++s)
            if (h->need_sol[s]) {
                if ((e = cudaMalloc(&h->DSOL[s], nval * sizeof(float))) != cudaSuccess) return cleanup_fail("sol alloc", e);
                h->device_bytes += nval * sizeof(float);
            }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cleanup_fail("setup", e);
    *out = h;
    return DGSW_OK;
}

// Autotuner: build the problem with each stage-kernel tile size, time a few steps of each on the
// device (after two warm-up steps that also capture the step graphs) and keep the fastest. `tune_*`
// describe the problem the timing runs on (a subset of an ensemble's members, or the problem itself);
// the winner is then built for the full problem unless the tuning problem is the full problem.
// Decisions are cached per (elements, order, precision, stages, options, device) for the process.
// an autotuner candidate and its device time per step; the decisions are cached per problem shape
struct TuneRecord {
    int tile, occ, order;
    double ms;
    int uncapped;
};
static std::mutex g_tune_mutex;
static std::map<std::string, TuneRecord> g_tune_cache;

// One tile size of the autotuner: a handle built with that tile, then each (occupancy, tile order) pair
// timed on it from the initial state: 2 warm-up steps, then graph-replayed steps worth about 2 ms (at
// least 4). Returns the handle (in *keep, left at the last variant) or destroys it.

static int32_t time_tile(const dgsw_config* cfg, const dgsw_mesh* mesh, const int32_t* group, int32_t ng,
                         const double* gp, int tile, std::vector<TuneRecord>& rec, dgsw_handle* keep) {
    dgsw_config c = *cfg;
    c.tile = tile;
    dgsw_handle h = nullptr;
    int32_t rc = create_impl(&c, mesh, group, ng, gp, &h);
    if (rc) return rc;
    const int warm = 2;
    for (int occ = 0; occ < 2; ++occ)
        for (int order = 0; order < 2; ++order) {
            destroy_graphs(h);  // the step graphs hold the kernel and its arguments
            h->occ = occ;
            h->order = order;
            if ((rc = dgsw_rkdg_init_state(h)) || (rc = dgsw_rkdg_step(h, warm))) {
                dgsw_rkdg_destroy(h);
                return rc;
            }
            // about 2 ms of timed steps (at least 4): on small meshes a few steps are launch-latency noise.
            // A batch of 8 or more replays 8-step graphs, captured here before the timed batch.
            double ms = 0;
            int64_t nl = 0;
            dgsw_rkdg_last_step_timing(h, &ms, &nl);
            const double est = ms / warm;
            const int timed = est > 0.0 ? std::max(4, std::min(256, (int)std::ceil(2.0 / est))) : 4;
            if ((timed >= 8 && (rc = dgsw_rkdg_step(h, 8))) || (rc = dgsw_rkdg_step(h, timed))) {
                dgsw_rkdg_destroy(h);
                return rc;
            }
            dgsw_rkdg_last_step_timing(h, &ms, &nl);
            rec.push_back({tile, occ, order, ms / timed, 0});
        }
    if (keep) {
        *keep = h;
    } else {
        dgsw_rkdg_destroy(h);
    }
    return DGSW_OK;
}

static int32_t create_tuned(const dgsw_config* cfg, const dgsw_mesh* mesh, const int32_t* group, int32_t ng,
                            const double* gp, const dgsw_mesh* tune_mesh, const int32_t* tune_group, int32_t tune_ng,
                            const double* tune_gp, dgsw_handle* out) {
    const bool same = tune_mesh == mesh;
    const int tiles[2] = {128, 256};
    cudaDeviceProp prop;
    std::memset(&prop, 0, sizeof(prop));
    cudaGetDeviceProperties(&prop, cfg->device);
    char key[512];
    std::snprintf(key, sizeof(key), "%lld/%lld/%d/%d/%d/%d/%d/%d/%d/%d/%d/%s", (long long)mesh->n_elems,
                  (long long)tune_mesh->n_elems, cfg->p, cfg->precision, cfg->rk_nstages, cfg->wetting_drying,
                  cfg->slope_limiting, cfg->function_source, cfg->bottom_friction, cfg->fp64_limiter, ng, prop.name);
    TuneRecord chosen = {0, 0, 0, 0.0, 0};
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) chosen = it->second;
    }
    std::vector<TuneRecord> rec;
    dgsw_handle kept[2] = {nullptr, nullptr};
    if (!chosen.tile) {
        for (int i = 0; i < 2; ++i) {
            int32_t rc = time_tile(cfg, tune_mesh, tune_group, tune_ng, tune_gp, tiles[i], rec, same ? &kept[i] : nullptr);
            if (rc) {
                for (dgsw_handle k : kept)
                    if (k) dgsw_rkdg_destroy(k);
                return rc;
            }
        }
        chosen = rec[0];
        for (const TuneRecord& r : rec)
            if (r.ms < chosen.ms) chosen = r;
        chosen.uncapped = -1;  // decided below, on the chosen configuration
    }
    dgsw_handle best = nullptr;
    for (int i = 0; i < 2; ++i) {
        if (kept[i] && tiles[i] == chosen.tile)
            best = kept[i];
        else if (kept[i])
            dgsw_rkdg_destroy(kept[i]);
    }
    if (!best) {
        dgsw_config c = *cfg;
        c.tile = chosen.tile;
        c.occupancy = chosen.occ;
        c.tile_order = chosen.order;
        int32_t rc = create_impl(&c, mesh, group, ng, gp, &best);
        if (rc) return rc;
        best->uncapped = chosen.uncapped > 0 ? 1 : 0;
    } else {
        destroy_graphs(best);
        best->occ = chosen.occ;
        best->order = chosen.order;
        best->uncapped = chosen.uncapped > 0 ? 1 : 0;
        int32_t rc = dgsw_rkdg_init_state(best);  // back to t = 0 after the timing steps
        if (rc) {
            dgsw_rkdg_destroy(best);
            return rc;
        }
    }
    if (chosen.uncapped < 0) {
        // the stage kernel's shared memory: where every tile fits the compile-time capacities, the capped
        // kernel and the kernel sized to the mesh's largest tile (less shared memory per SM, so a larger L1)
        // are timed alternately, 3 rounds of 8 graph-replayed steps each after 8 warm-up steps, and the
        // faster kept. Measured per step: sized to the mesh, config 2 runs 1.5 % (FP32) and 4.9 % (FP64)
        // faster and the p = 2 tidal channel 6.9 % (FP64); the p = 1 bowl stays capped (7 % slower sized).
        chosen.uncapped = 0;
        if (stage_fits_caps(best->tile, best->tiling.max_halo, best->tiling.max_edges)) {
            double t[2] = {0.0, 0.0};
            bool ok = true;
            for (int round = 0; round < 3 && ok; ++round)
                for (int i = 0; i < 2 && ok; ++i) {
                    const int unc = (round & 1) ? 1 - i : i;
                    destroy_graphs(best);
                    best->uncapped = unc;
                    // a problem that fails within these 16 steps keeps the capped kernel; the failure
                    // is then the caller's to meet in its own steps
                    ok = !dgsw_rkdg_init_state(best) && !dgsw_rkdg_step(best, 8) && !dgsw_rkdg_step(best, 8);
                    double ms = 0;
                    int64_t nl = 0;
                    if (ok) dgsw_rkdg_last_step_timing(best, &ms, &nl);
                    t[unc] += ms;
                }
            chosen.uncapped = ok && t[1] < t[0] ? 1 : 0;
            destroy_graphs(best);
            best->uncapped = chosen.uncapped;
            int32_t rc = dgsw_rkdg_init_state(best);
            if (rc) {
                dgsw_rkdg_destroy(best);
                return rc;
            }
        }
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        g_tune_cache[key] = chosen;
    }
    best->n_tuned = (int32_t)std::min<size_t>(rec.size(), DGSW_TUNE_MAX_CANDIDATES);
    for (int i = 0; i < best->n_tuned; ++i) {
        best->tuned_tile[i] = rec[i].tile;
        best->tuned_occ[i] = rec[i].occ;
        best->tuned_order[i] = rec[i].order;
        best->tuned_ms[i] = rec[i].ms;
    }
    *out = best;
    return DGSW_OK;
}

int32_t dgsw_rkdg_create(const dgsw_config* cfg, const dgsw_mesh* mesh, dgsw_handle* out) {
    if (!cfg || !mesh || !out) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    if (cfg->tile == DGSW_TILE_AUTOTUNE) return create_tuned(cfg, mesh, nullptr, 0, nullptr, mesh, nullptr, 0, nullptr, out);
    return create_impl(cfg, mesh, nullptr, 0, nullptr, out);
}

// members -> one mesh: nodes and boundary chains appended with index offsets, element IDs renumbered
// member-major (ascending within each member by its own IDs), caller_group = member of each element
struct Concat {
    std::vector<double> xyz, manning;
    std::vector<int32_t> en, seg_type, seg_nodes, group;
    std::vector<uint32_t> ids;
    std::vector<int64_t> seg_off{0};
    std::vector<std::vector<int32_t>> fnodes;  // forcing block nodes, offset to the joint numbering
    std::vector<dgsw_forcing_block> forcing;
    std::vector<int32_t> levee_nodes;          // levee pairs, offset to the joint numbering
    std::vector<double> levee_data;
    dgsw_mesh m{};
};

static int concat_members(int32_t n, const dgsw_mesh* members, Concat& C, std::string& err) {
    int64_t nn = 0, ne = 0;
    for (int32_t k = 0; k < n; ++k) {
        const dgsw_mesh& M = members[k];
        if (!M.node_xyz || !M.elem_nodes || M.n_nodes <= 0 || M.n_elems <= 0 || (M.n_segments && !M.seg_offsets)) {
            err = "ensemble member " + std::to_string(k) + " has no nodes or elements";
            return DGSW_ERR_INVALID_ARGUMENT;
        }
        nn += M.n_nodes;
        ne += M.n_elems;
    }
    if (ne >= ((int64_t)1 << 32) || nn >= ((int64_t)1 << 31)) {
        err = "ensemble too large for 32-bit element IDs";
        return DGSW_ERR_UNSUPPORTED;
    }
    C.xyz.reserve(3 * nn);
    C.en.reserve(3 * ne);
    C.ids.reserve(ne);
    C.group.reserve(ne);
    int64_t node_base = 0, id_base = 0;
    for (int32_t k = 0; k < n; ++k) {
        const dgsw_mesh& M = members[k];
        C.xyz.insert(C.xyz.end(), M.node_xyz, M.node_xyz + 3 * M.n_nodes);
        std::vector<int64_t> order(M.n_elems);
        std::iota(order.begin(), order.end(), 0);
        if (M.elem_ids)
            std::stable_sort(order.begin(), order.end(),
                             [&](int64_t a, int64_t b) { return M.elem_ids[a] < M.elem_ids[b]; });
        std::vector<uint32_t> rank(M.n_elems);
        for (int64_t i = 0; i < M.n_elems; ++i) rank[order[i]] = (uint32_t)(id_base + i);
        for (int64_t i = 0; i < M.n_elems; ++i) {
            for (int v = 0; v < 3; ++v) {
                const int32_t nd = M.elem_nodes[3 * i + v];
                if (nd < 0 || nd >= M.n_nodes) {
                    err = "ensemble member " + std::to_string(k) + ": element node index out of range";
                    return DGSW_ERR_MESH;
                }
                C.en.push_back((int32_t)(nd + node_base));
            }
            C.ids.push_back(rank[i]);
            C.group.push_back(k);
        }
        for (int32_t sgm = 0; sgm < M.n_segments; ++sgm) {
            C.seg_type.push_back(M.seg_type[sgm]);
            for (int64_t i = M.seg_offsets[sgm]; i < M.seg_offsets[sgm + 1]; ++i)
                C.seg_nodes.push_back((int32_t)(M.seg_nodes[i] + node_base));
            C.seg_off.push_back((int64_t)C.seg_nodes.size());
        }
        if (M.node_manning_n) {
            C.manning.resize(node_base, 0.0);
            C.manning.insert(C.manning.end(), M.node_manning_n, M.node_manning_n + M.n_nodes);
        }
        if (M.n_forcing > 0 && !M.forcing) {
            err = "ensemble member " + std::to_string(k) + ": null forcing block list";
            return DGSW_ERR_INVALID_ARGUMENT;
        }
        // a member's blocks hold only its own nodes, so its faces find only its own blocks
        for (int32_t b = 0; b < M.n_forcing; ++b) {
            const dgsw_forcing_block& B = M.forcing[b];
            if (B.n_nodes > 0 && !B.nodes) {
                err = "ensemble member " + std::to_string(k) + ": forcing block without nodes";
                return DGSW_ERR_INVALID_ARGUMENT;
            }
            std::vector<int32_t> nodes((size_t)std::max(B.n_nodes, 0));
            for (int32_t j = 0; j < B.n_nodes; ++j) {
                if (B.nodes[j] < 0 || B.nodes[j] >= M.n_nodes) {
                    err = "ensemble member " + std::to_string(k) + ": forcing node index out of range";
                    return DGSW_ERR_MESH;
                }
                nodes[j] = (int32_t)(B.nodes[j] + node_base);
            }
            C.fnodes.push_back(std::move(nodes));
            C.forcing.push_back(B);
        }
        if (M.n_levee_pairs > 0 && (!M.levee_nodes || !M.levee_data)) {
            err = "ensemble member " + std::to_string(k) + ": null levee pair list";
            return DGSW_ERR_INVALID_ARGUMENT;
        }
        for (int32_t i = 0; i < M.n_levee_pairs; ++i) {
            for (int j = 0; j < 2; ++j) {
                const int32_t n = M.levee_nodes[2 * i + j];
                if (n < 0 || n >= M.n_nodes) {
                    err = "ensemble member " + std::to_string(k) + ": levee node index out of range";
                    return DGSW_ERR_MESH;
                }
                C.levee_nodes.push_back((int32_t)(n + node_base));
            }
            for (int j = 0; j < 3; ++j) C.levee_data.push_back(M.levee_data[3 * i + j]);
        }
        node_base += M.n_nodes;
        id_base += M.n_elems;
    }
    C.m.n_nodes = nn;
    C.m.node_xyz = C.xyz.data();
    C.m.n_elems = ne;
    C.m.elem_nodes = C.en.data();
    C.m.elem_ids = C.ids.data();
    C.m.n_segments = (int32_t)C.seg_type.size();
    C.m.seg_type = C.seg_type.data();
    C.m.seg_offsets = C.seg_off.data();
    C.m.seg_nodes = C.seg_nodes.data();
    if (!C.manning.empty()) {
        C.manning.resize(nn, 0.0);
        C.m.node_manning_n = C.manning.data();
    }
    for (size_t b = 0; b < C.forcing.size(); ++b) C.forcing[b].nodes = C.fnodes[b].data();
    C.m.n_forcing = (int32_t)C.forcing.size();
    C.m.forcing = C.forcing.empty() ? nullptr : C.forcing.data();
    C.m.n_levee_pairs = (int32_t)(C.levee_nodes.size() / 2);
    C.m.levee_nodes = C.levee_nodes.empty() ? nullptr : C.levee_nodes.data();
    C.m.levee_data = C.levee_data.empty() ? nullptr : C.levee_data.data();
    return DGSW_OK;
}

int32_t dgsw_ensemble_create(const dgsw_config* cfg, int32_t n_members, const dgsw_mesh* members,
                             const double* member_params, dgsw_handle* out) {
    if (!cfg || !members || !out || n_members < 1) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument or no members");
    *out = nullptr;
    std::vector<double> params((size_t)n_members * DGSW_FN_PARAMS);
    for (int32_t k = 0; k < n_members; ++k)
        for (int i = 0; i < DGSW_FN_PARAMS; ++i)
            params[(size_t)k * DGSW_FN_PARAMS + i] =
                member_params ? member_params[(size_t)k * DGSW_FN_PARAMS + i] : cfg->fn_params[i];
    Concat all;
    std::string err;
    int rc = concat_members(n_members, members, all, err);
    if (rc) return fail(rc, err);
    if (cfg->tile != DGSW_TILE_AUTOTUNE) return create_impl(cfg, &all.m, all.group.data(), n_members, params.data(), out);
    // tune on the leading members, up to about 2^19 elements (all of them for a small ensemble)
    int32_t nt = 0;
    int64_t acc = 0;
    while (nt < n_members && (nt == 0 || acc + members[nt].n_elems <= ((int64_t)1 << 19))) acc += members[nt++].n_elems;
    if (nt == n_members)
        return create_tuned(cfg, &all.m, all.group.data(), n_members, params.data(), &all.m, all.group.data(),
                            n_members, params.data(), out);
    Concat sub;
    if ((rc = concat_members(nt, members, sub, err))) return fail(rc, err);
    return create_tuned(cfg, &all.m, all.group.data(), n_members, params.data(), &sub.m, sub.group.data(), nt,
                        params.data(), out);
}

int32_t dgsw_ensemble_member_range(dgsw_handle h, int32_t member, int64_t* first, int64_t* n_elems) {
    if (!h || !first || !n_elems) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    if (h->member_first.empty()) {
        if (member != 0) return fail(DGSW_ERR_INVALID_ARGUMENT, "not an ensemble: only member 0 exists");
        *first = 0;
        *n_elems = h->ne;
        return DGSW_OK;
    }
    if (member < 0 || member >= h->n_members) return fail(DGSW_ERR_INVALID_ARGUMENT, "member index out of range");
    *first = h->member_first[member];
    *n_elems = h->member_first[member + 1] - h->member_first[member];
    return DGSW_OK;
}

int32_t dgsw_rkdg_tuning(dgsw_handle h, int32_t* tiles, int32_t* occupancy, int32_t* tile_order, double* ms_per_step,
                         int32_t* n) {
    if (!h || !n) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    *n = h->n_tuned;
    for (int i = 0; i < h->n_tuned; ++i) {
        if (tiles) tiles[i] = h->tuned_tile[i];
        if (occupancy) occupancy[i] = h->tuned_occ[i];
        if (tile_order) tile_order[i] = h->tuned_order[i];
        if (ms_per_step) ms_per_step[i] = h->tuned_ms[i];
    }
    return DGSW_OK;
}

int32_t dgsw_rkdg_destroy(dgsw_handle h) {
    if (!h) return DGSW_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroy_graphs(h);
    for (void* p : h->Q)
        if (p) cudaFree(p);
    for (void* p : h->SOL)
        if (p) cudaFree(p);
    for (void* p : h->D)
        if (p) cudaFree(p);
    for (void* p : h->DSOL)
        if (p) cudaFree(p);
    for (void* p : h->QF)
        if (p) cudaFree(p);
    for (void* p : h->QL)
        if (p) cudaFree(p);
    if (h->bath) cudaFree(h->bath);
    if (h->geo) cudaFree(h->geo);
    if (h->egeo) cudaFree(h->egeo);
    if (h->manning) cudaFree(h->manning);
    h->fface.release();
    h->fcon.release();
    h->lev.release();
    h->ldat.release();
    h->levF.release();
    h->went_dry.release();
    h->post.release();
    h->post_flags.release();
    h->halo.release();
    h->tile_halo_off.release();
    h->enodes.release();
    h->tile_edge_off.release();
    h->ref_of_dev.release();
    h->eslot.release();
    h->edges.release();
    h->xy.release();
    h->nz.release();
    h->wet[0].release();
    h->wet[1].release();
    h->status.release();
    h->clock.release();
    h->red.release();
    h->l2rule.release();
    h->staging.release();
    h->limited.release();
    h->nbr.release();
    h->baryctr.release();
    h->lgeo.release();
    h->lgeo_f.release();
    h->nbr_face.release();
    h->tI.release();
    h->tflag.release();
    h->tscratch.release();
    h->tout.release();
    h->ind_params.release();
    h->ind_list.release();
    h->ind_count.release();
    h->ind_gate.release();
    h->ind_counters.release();
    h->ind_error.release();
    for (cudaEvent_t ev : h->kt_ev) cudaEventDestroy(ev);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return DGSW_OK;
}

int32_t dgsw_rkdg_info(dgsw_handle h, dgsw_info* o) {
    if (!h || !o) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(o, 0, sizeof(*o));
    o->n_elems = h->ne;
    o->n_nodes = h->nn;
    o->n_interfaces = (int64_t)h->topo.intf.size() / 4;
    o->n_boundaries = (int64_t)h->topo.bnd.size() / 3;
    o->n_tiles = h->tiling.ntiles;
    o->n_tile_edges = (int64_t)h->tiling.edges.size() / 4;
    o->p = h->cfg.p;
    o->ndof = h->nd;
    o->ngp_volume = h->tb.nq;
    o->ngp_edge = h->tb.ng;
    o->nstages = h->ns;
    o->precision = h->cfg.precision;
    o->tile = h->tile;
    o->device_bytes = h->device_bytes;
    o->state_bytes = (int64_t)3 * h->nd * h->ne_pad * (int64_t)sizeof(double);
    o->occupancy = h->occ;
    o->tile_order = h->order;
    o->stage_increments = h->split ? 1 : 0;
    o->smem_capped = (!h->uncapped && stage_fits_caps(h->tile, h->tiling.max_halo, h->tiling.max_edges)) ? 1 : 0;
    return DGSW_OK;
}

int32_t dgsw_rkdg_init_state(dgsw_handle h) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    cudaSetDevice(h->device);
    std::vector<double> q;
    project_initial_condition(h->topo, h->node_xyz.data(), h->tb, h->cfg, q);
    std::vector<uint8_t> wet;
    init_wet_dry(h->topo, h->node_xyz.data(), h->tb, h->cfg, q, wet);
    h->t = 0.0;
    h->step = 0;
    h->stage = 0;
    DevClock c = {0.0, 0};
    CUDA_TRY(cudaMemcpyAsync(h->clock.p, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    int rc = upload_state(h, q.data());
    if (rc) return rc;
    return upload_wet(h, wet.data());
}

int32_t dgsw_rkdg_set_state(dgsw_handle h, const double* q) {
    if (!h || !q) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    return upload_state(h, q);
}

int32_t dgsw_rkdg_get_state(dgsw_handle h, double* q) {
    if (!h || !q) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    return download_state(h, q);
}

int32_t dgsw_rkdg_postprocess(dgsw_handle h, double* point_data, double* cell_data, uint8_t* wet, uint8_t* went_dry) {
    if (!h || !point_data || !cell_data) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    cudaError_t e;
    if (!h->post.p) {
        if ((e = h->post.alloc((size_t)h->ne * 16)) != cudaSuccess || (e = h->post_flags.alloc((size_t)h->ne * 2)) != cudaSuccess)
            return fail(DGSW_ERR_CUDA, std::string("postprocess buffers: ") + cudaGetErrorString(e));
        h->device_bytes += h->ne * 130;
    }
    // the master element's modes at the VTK points (Triangle::VTKPostPoint / VTKPostCell, N_DIV = 1)
    const double dz = 2.0;
    const double z1[4] = {-1.0, -1.0 + dz, -1.0, -1.0 + dz / 3.0};
    const double z2[4] = {-1.0, -1.0, -1.0 + dz, -1.0 + dz / 3.0};
    double phi[6 * 4];
    eval_basis(h->cfg.p, z1, z2, 4, phi);
    auto run = [&](auto bath_ptr) {
        using R = typename std::remove_cv<typename std::remove_pointer<decltype(bath_ptr)>::type>::type;
        PostArgs<R> A;
        std::memset(&A, 0, sizeof(A));
        A.q = (const double*)h->Q[h->stage];
        A.bath = bath_ptr;
        A.wet = h->wet[h->wet_cur].p;
        A.went_dry = h->went_dry.p;
        A.ref_of_dev = h->ref_of_dev.p;
        for (int pt = 0; pt < 4; ++pt)
            for (int k = 0; k < h->nd; ++k) A.phi[pt][k] = phi[k * 4 + pt];
        A.point = h->post.p;
        A.cell = h->post.p + (size_t)h->ne * 12;
        A.wet_out = h->post_flags.p;
        A.went_dry_out = h->post_flags.p + h->ne;
        A.ne = (int)h->ne;
        A.ne_pad = (int)h->ne_pad;
        A.nd = h->nd;
        return launch_postprocess<R>(A, h->stream);
    };
    e = split_form(h, h->stage);
    if (e == cudaSuccess) e = h->fp32 ? run((const float*)h->bath) : run((const double*)h->bath);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("postprocess: ") + cudaGetErrorString(e));
    CUDA_TRY(cudaMemcpyAsync(point_data, h->post.p, (size_t)h->ne * 12 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(cell_data, h->post.p + (size_t)h->ne * 12, (size_t)h->ne * 4 * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
    if (wet) CUDA_TRY(cudaMemcpyAsync(wet, h->post_flags.p, (size_t)h->ne, cudaMemcpyDeviceToHost, h->stream));
    if (went_dry)
        CUDA_TRY(cudaMemcpyAsync(went_dry, h->post_flags.p + h->ne, (size_t)h->ne, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

int32_t dgsw_rkdg_get_bathymetry(dgsw_handle h, double* modes) {
    if (!h || !modes) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<double> b;
    project_bathymetry(h->topo, h->node_xyz.data(), h->tb, b);
    std::memcpy(modes, b.data(), b.size() * sizeof(double));
    return DGSW_OK;
}

int32_t dgsw_rkdg_set_wet(dgsw_handle h, const uint8_t* wet) {
    if (!h || !wet) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    return upload_wet(h, wet);
}

int32_t dgsw_rkdg_get_wet(dgsw_handle h, uint8_t* wet) {
    if (!h || !wet) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    std::vector<unsigned char> w(h->ne_pad);
    CUDA_TRY(cudaMemcpyAsync(w.data(), h->wet[h->wet_cur].p, h->ne_pad, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t d = 0; d < h->ne; ++d) wet[h->tiling.ref_of_dev[d]] = w[d];
    return DGSW_OK;
}

int32_t dgsw_rkdg_get_limited(dgsw_handle h, uint8_t* flags) {
    if (!h || !flags) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    std::vector<unsigned char> w(h->ne_pad);
    CUDA_TRY(cudaMemcpyAsync(w.data(), h->limited.p, h->ne_pad, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t d = 0; d < h->ne; ++d) flags[h->tiling.ref_of_dev[d]] = w[d];
    return DGSW_OK;
}

int32_t dgsw_rkdg_indicator_features(dgsw_handle h, float* d_features, uint8_t* d_ok) {
    if (!h || !d_features) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    if (h->cfg.p != 1) return fail(DGSW_ERR_UNSUPPORTED, "the troubled-cell indicator is defined for p = 1");
    cudaSetDevice(h->device);
    cudaError_t e = split_form(h, h->stage);
    if (e == cudaSuccess)
        e = launch_indicator_features<double>(feature_args<double>(h, h->stage), h->ref_of_dev.p, d_features, d_ok,
                                              h->stream);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("indicator features: ") + cudaGetErrorString(e));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

int32_t dgsw_rkdg_stage_record(dgsw_handle h, float* d_features, uint8_t* d_labels) {
    if (!h || !d_features || !d_labels) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    if (h->cfg.p != 1) return fail(DGSW_ERR_UNSUPPORTED, "the troubled-cell indicator is defined for p = 1");
    cudaSetDevice(h->device);
    int64_t launches = 0;
    StageRecord rec{d_features, d_labels};
    cudaError_t e = enqueue_stage(h, h->stage, launches, &rec);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("stage: ") + cudaGetErrorString(e));
    advance_host_stepper(h);
    return check_status(h);
}

int32_t dgsw_rkdg_set_indicator(dgsw_handle h, const float* params, double confidence, int32_t mode) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (mode < 0 || mode > 2) return fail(DGSW_ERR_INVALID_ARGUMENT, "indicator mode must be 0, 1 or 2");
    cudaSetDevice(h->device);
    if (mode == 0) {
        if (h->ind_mode != 0) destroy_graphs(h);
        h->ind_mode = 0;
        return DGSW_OK;
    }
    if (!params) return fail(DGSW_ERR_INVALID_ARGUMENT, "null indicator parameters");
    if (!h->cfg.slope_limiting) return fail(DGSW_ERR_INVALID_ARGUMENT, "the indicator gates the slope limiter, "
                                                                       "which this problem does not use");
    if (h->cfg.p != 1) return fail(DGSW_ERR_UNSUPPORTED, "the troubled-cell indicator is defined for p = 1");
    if (!(confidence >= 0.5 && confidence <= 1.0))
        return fail(DGSW_ERR_INVALID_ARGUMENT, "indicator confidence must lie in [0.5, 1]");
    cudaError_t e;
    if (!h->ind_params.p) {
        if ((e = h->ind_params.alloc(MLP_NPARAM)) != cudaSuccess ||
            (e = h->ind_list.alloc(h->ne_pad)) != cudaSuccess || (e = h->ind_count.alloc(1)) != cudaSuccess ||
            (e = h->ind_gate.alloc(h->ne_pad)) != cudaSuccess ||
            (e = h->ind_counters.alloc(IND_NCOUNTERS)) != cudaSuccess || (e = h->ind_error.alloc(1)) != cudaSuccess)
            return fail(DGSW_ERR_CUDA, std::string("indicator buffers: ") + cudaGetErrorString(e));
        h->device_bytes += (int64_t)MLP_NPARAM * 4 + h->ne_pad * 5 + 64;
        CUDA_TRY(cudaMemsetAsync(h->ind_counters.p, 0, IND_NCOUNTERS * sizeof(unsigned long long), h->stream));
        CUDA_TRY(cudaMemsetAsync(h->ind_error.p, 0, sizeof(int), h->stream));
        CUDA_TRY(cudaMemsetAsync(h->ind_count.p, 0, sizeof(int), h->stream));
    }
    CUDA_TRY(cudaMemcpyAsync(h->ind_params.p, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->ind_mode != mode) destroy_graphs(h);
    h->ind_mode = mode;
    h->ind_skip_below = (float)(1.0 - confidence);
    return DGSW_OK;
}

int32_t dgsw_rkdg_set_indicator_features(dgsw_handle h, int32_t feature_set) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (feature_set != IND_FEATURES_CHARACTERISTIC && feature_set != IND_FEATURES_RAW)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "feature set must be 0 (characteristic) or 1 (raw)");
    h->ind_fset = feature_set;
    destroy_graphs(h);  // a gated step graph holds the feature arguments
    return DGSW_OK;
}

int32_t dgsw_rkdg_indicator_stats(dgsw_handle h, int64_t* counts, int32_t reset) {
    if (!h || !counts) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < 4; ++i) counts[i] = 0;
    if (!h->ind_counters.p) return DGSW_OK;
    cudaSetDevice(h->device);
    unsigned long long c[IND_NCOUNTERS];
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(c, h->ind_counters.p, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(&err, h->ind_error.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < 4; ++i) counts[i] = (int64_t)c[i];
    if (reset) {
        CUDA_TRY(cudaMemsetAsync(h->ind_counters.p, 0, sizeof(c), h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    if (err) return fail(DGSW_ERR_CUDA, "indicator: a tensor-core wait timed out");
    return DGSW_OK;
}

int32_t dgsw_rkdg_set_trouble(dgsw_handle h, int32_t enable) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (enable && !h->cfg.slope_limiting)
        return fail(DGSW_ERR_INVALID_ARGUMENT, "the trouble indicator belongs to the slope limiter, which this "
                                               "problem does not use");
    cudaSetDevice(h->device);
    if (enable && !h->tI.p) {
        cudaError_t e;
        std::vector<signed char> nf((size_t)3 * h->ne_pad, -1);
        for (int64_t d = 0; d < h->ne; ++d) {
            const int64_t r = h->tiling.ref_of_dev[d];
            for (int f = 0; f < 3; ++f) nf[(size_t)f * h->ne_pad + d] = h->topo.nbr_face[3 * r + f];
        }
        if ((e = h->nbr_face.alloc(nf.size())) != cudaSuccess || (e = h->tI.alloc(h->ne_pad)) != cudaSuccess ||
            (e = h->tflag.alloc(h->ne_pad)) != cudaSuccess || (e = h->tscratch.alloc(h->ne_pad)) != cudaSuccess ||
            (e = h->tout.alloc(h->ne_pad)) != cudaSuccess)
            return fail(DGSW_ERR_CUDA, std::string("trouble buffers: ") + cudaGetErrorString(e));
        CUDA_TRY(cudaMemcpy(h->nbr_face.p, nf.data(), nf.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemset(h->tI.p, 0, h->ne_pad * sizeof(double)));
        CUDA_TRY(cudaMemset(h->tout.p, 0, h->ne_pad));
        h->device_bytes += (int64_t)h->ne_pad * 14;
    }
    if ((enable != 0) != (h->trouble_on != 0)) destroy_graphs(h);
    h->trouble_on = enable != 0;
    return DGSW_OK;
}

int32_t dgsw_rkdg_get_trouble(dgsw_handle h, double* I, uint8_t* troubled) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (!h->tI.p) return fail(DGSW_ERR_INVALID_ARGUMENT, "the trouble indicator is not enabled");
    cudaSetDevice(h->device);
    std::vector<double> v(h->ne);
    std::vector<unsigned char> t(h->ne);
    CUDA_TRY(cudaMemcpyAsync(v.data(), h->tI.p, h->ne * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(t.data(), h->tout.p, h->ne, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t d = 0; d < h->ne; ++d) {
        const int64_t r = h->tiling.ref_of_dev[d];
        if (I) I[r] = v[d];
        if (troubled) troubled[r] = t[d];
    }
    return DGSW_OK;
}

int32_t dgsw_rkdg_set_state_device(dgsw_handle h, const void* d_q) {
    if (!h || !d_q) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    cudaError_t e = launch_permute_in<double, double>((const double*)d_q, (double*)h->Q[h->stage], h->ref_of_dev.p,
                                                      (int)h->ne, (int)h->ne_pad, 3 * h->nd, h->stream);
    if (e == cudaSuccess) e = split_absorb(h);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("set_state_device: ") + cudaGetErrorString(e));
    return DGSW_OK;
}

int32_t dgsw_rkdg_get_state_device(dgsw_handle h, void* d_q) {
    if (!h || !d_q) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    cudaError_t e = split_form(h, h->stage);
    if (e == cudaSuccess)
        e = launch_permute_out<double, double>((const double*)h->Q[h->stage], (double*)d_q, h->ref_of_dev.p,
                                               (int)h->ne, (int)h->ne_pad, 3 * h->nd, h->stream);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("get_state_device: ") + cudaGetErrorString(e));
    return DGSW_OK;
}

int32_t dgsw_rkdg_stage(dgsw_handle h) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    cudaSetDevice(h->device);
    int64_t launches = 0;
    cudaError_t e = enqueue_stage(h, h->stage, launches);
    if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("stage: ") + cudaGetErrorString(e));
    advance_host_stepper(h);
    return check_status(h);
}

int32_t dgsw_rkdg_step(dgsw_handle h, int32_t nsteps) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (nsteps < 0) return fail(DGSW_ERR_INVALID_ARGUMENT, "negative step count");
    cudaSetDevice(h->device);
    int64_t launches = 0;
    CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    // finish a partially advanced step stage by stage
    while (h->stage != 0 && nsteps > 0) {
        cudaError_t e = enqueue_stage(h, h->stage, launches);
        if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("stage: ") + cudaGetErrorString(e));
        advance_host_stepper(h);
        if (h->stage == 0) --nsteps;
    }
    for (int32_t n = 0; n < nsteps;) {
        // a captured step bakes in the buffer pointers: key the graphs by the parity of the
        // q_0 <-> q_ns swaps and by which wet-flag buffer is current
        const int key = h->qswap + 2 * h->wet_cur;
        if (h->cfg.use_graphs) {
            const int m = nsteps - n >= GRAPH_MULTI ? GRAPH_MULTI : 1;  // steps in this graph
            cudaGraphExec_t& gx = m > 1 ? h->graph_multi[key] : h->graph[key];
            int64_t& gl = m > 1 ? h->graph_multi_launches[key] : h->graph_launches[key];
            if (!gx) {
                cudaGraph_t g;
                std::vector<void*> Qsave = h->Q;
                const int wsave = h->wet_cur, qsave = h->qswap;
                CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
                int64_t l2 = 0;
                cudaError_t ce = cudaSuccess;
                for (int s = 0; s < m * h->ns && ce == cudaSuccess; ++s) ce = enqueue_stage(h, s % h->ns, l2);
                cudaError_t ee = cudaStreamEndCapture(h->stream, &g);
                h->Q = Qsave;
                h->wet_cur = wsave;
                h->qswap = qsave;
                if (ce != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
                if (ee != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("capture end: ") + cudaGetErrorString(ee));
                CUDA_TRY(cudaGraphInstantiate(&gx, g, 0));
                cudaGraphDestroy(g);
                gl = l2;
            }
            CUDA_TRY(cudaGraphLaunch(gx, h->stream));
            launches += gl;
            // replay the host-side buffer rotation of the graph's steps
            for (int s = 0; s < m * h->ns; ++s) {
                h->wet_cur = 1 - h->wet_cur;
                if ((s + 1) % h->ns == 0) {
                    std::swap(h->Q[0], h->Q[h->ns]);
                    h->qswap ^= 1;
                }
            }
            for (int s = 0; s < m * h->ns; ++s) advance_host_stepper(h);
            n += m;
        } else {
            for (int s = 0; s < h->ns; ++s) {
                cudaError_t e = enqueue_stage(h, s, launches);
                if (e != cudaSuccess) return fail(DGSW_ERR_CUDA, std::string("stage: ") + cudaGetErrorString(e));
            }
            for (int s = 0; s < h->ns; ++s) advance_host_stepper(h);
            ++n;
        }
    }
    CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    int rc = check_status(h);
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_ms = ms;
    h->last_launches = launches;
    return rc;
}

int32_t dgsw_rkdg_step_timed(dgsw_handle h, int32_t nsteps, double* stage_ms, int64_t* stage_launches) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (nsteps < 0 || nsteps > 100000) return fail(DGSW_ERR_INVALID_ARGUMENT, "step count out of range");
    cudaSetDevice(h->device);
    // one event pair per stage of the batch, created once and kept for later calls
    const size_t need = 2 * (size_t)(nsteps + 1) * (size_t)h->ns;
    while (h->kt_ev.size() < need) {
        cudaEvent_t ev;
        CUDA_TRY(cudaEventCreate(&ev));
        h->kt_ev.push_back(ev);
    }
    // the stages run as separate launches (no step graphs), each bracketed by its own events
    const int32_t graphs = h->cfg.use_graphs;
    h->cfg.use_graphs = 0;
    h->kt_on = true;
    h->kt_used = 0;
    const int32_t rc = dgsw_rkdg_step(h, nsteps);
    h->kt_on = false;
    h->cfg.use_graphs = graphs;
    if (rc != DGSW_OK) return rc;
    double total = 0.0;
    for (size_t i = 0; i + 1 < h->kt_used; i += 2) {
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, h->kt_ev[i], h->kt_ev[i + 1]));
        total += ms;
    }
    if (stage_ms) *stage_ms = total;
    if (stage_launches) *stage_launches = (int64_t)(h->kt_used / 2);
    return DGSW_OK;
}

int32_t dgsw_rkdg_get_time(dgsw_handle h, double* t, int64_t* step, int32_t* stage) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (t) *t = h->t + h->cfg.dt * h->rk.drk[h->stage];
    if (step) *step = h->step;
    if (stage) *stage = h->stage;
    return DGSW_OK;
}

int32_t dgsw_rkdg_l2_error(dgsw_handle h, double* out) {
    if (!h || !out) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    double s = 0;
    int rc = h->fp32 ? run_reduction<float>(h, 0, &s) : run_reduction<double>(h, 0, &s);
    if (rc) return rc;
    *out = std::sqrt(s);
    return DGSW_OK;
}

int32_t dgsw_rkdg_mass(dgsw_handle h, double* out) {
    if (!h || !out) return fail(DGSW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(h->device);
    return h->fp32 ? run_reduction<float>(h, 1, out) : run_reduction<double>(h, 1, out);
}

int32_t dgsw_rkdg_topology(dgsw_handle h, int32_t* neighbors, uint8_t* btype, int64_t* n_interfaces,
                           int32_t* interfaces, int64_t* n_boundaries, int32_t* boundaries) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    const Topology& T = h->topo;
    if (neighbors) std::memcpy(neighbors, T.nbr.data(), T.nbr.size() * sizeof(int32_t));
    if (btype) std::memcpy(btype, T.btype.data(), T.btype.size());
    if (n_interfaces) *n_interfaces = (int64_t)T.intf.size() / 4;
    if (interfaces) std::memcpy(interfaces, T.intf.data(), T.intf.size() * sizeof(int32_t));
    if (n_boundaries) *n_boundaries = (int64_t)T.bnd.size() / 3;
    if (boundaries) std::memcpy(boundaries, T.bnd.data(), T.bnd.size() * sizeof(int32_t));
    return DGSW_OK;
}

int32_t dgsw_mesh_topology(const dgsw_mesh* mesh, int32_t* neighbors, uint8_t* btype, int64_t* n_interfaces,
                           int32_t* interfaces, int64_t* n_boundaries, int32_t* boundaries) {
    if (!mesh) return fail(DGSW_ERR_INVALID_ARGUMENT, "null mesh");
    Topology T;
    std::string err;
    int rc = build_topology(mesh, T, err);
    if (rc) return fail(rc, err);
    if (neighbors) std::memcpy(neighbors, T.nbr.data(), T.nbr.size() * sizeof(int32_t));
    if (btype) std::memcpy(btype, T.btype.data(), T.btype.size());
    if (n_interfaces) *n_interfaces = (int64_t)T.intf.size() / 4;
    if (interfaces) std::memcpy(interfaces, T.intf.data(), T.intf.size() * sizeof(int32_t));
    if (n_boundaries) *n_boundaries = (int64_t)T.bnd.size() / 3;
    if (boundaries) std::memcpy(boundaries, T.bnd.data(), T.bnd.size() * sizeof(int32_t));
    return DGSW_OK;
}

int32_t dgsw_rkdg_set_stream(dgsw_handle h, void* s) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)s;
    h->own_stream = false;
    destroy_graphs(h);
    return DGSW_OK;
}

int32_t dgsw_rkdg_synchronize(dgsw_handle h) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    cudaSetDevice(h->device);
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DGSW_OK;
}

int32_t dgsw_rkdg_last_step_timing(dgsw_handle h, double* ms, int64_t* launches) {
    if (!h) return fail(DGSW_ERR_INVALID_ARGUMENT, "null handle");
    if (ms) *ms = h->last_ms;
    if (launches) *launches = h->last_launches;
    return DGSW_OK;
}

}  // extern "C"
