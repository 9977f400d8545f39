// Allocation-free L2 error of a caller-owned FP64 state: dgsw_l2_error_static.
//
// Who needs it: a driver that hands all of the GPU's memory to its own pool before the run starts
// (an ensemble or coupled-model driver on PyTorch's caching allocator, or on a coupler's arena) cannot
// let a library cudaMalloc in the middle of the run: the call fails once the pool holds the memory, or
// takes memory the pool counted on. A monitoring loop that checks the error between asynchronously
// queued steps also avoids cudaMalloc/cudaFree, because they can synchronise the device and stall the
// queued work. This entry point allocates nothing: its scratch is the file-scope array below, whose
// memory the CUDA runtime reserves when it loads this module onto a device.
//
// Math: the same per-element sum as the handle's L2 error (Simulation::ComputeL2Residual,
// source/simulation/serial/simulation.hpp:85-93, with Element::ComputeResidualL2,
// source/geometry/element.hpp:549-592) with the degree-20 collapsed product rule; only the summation
// order differs (ascending element order here, tile order in the handle).
//
// Scratch use per call: kernel 1 writes one partial per 256-element block into scratch[0, nblocks);
// kernel 2 adds those partials in a fixed order into scratch[DGSW_L2_STATIC_MAX_ELEMS / 256]; the host
// copies that one slot back. Every slot that is read is written earlier in the same call, so nothing
// needs to start at zero and nothing is cleared. All calls on a device share the array: calls whose
// kernels overlap on the GPU (two host threads, or two streams without ordering between them) race on
// it and may return each other's sums.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dgsw_rkdg.h"
#include "function_sets.h"
#include "host_setup.h"
#include "quadrature.h"
#include "reduce_kernels.cuh"

using namespace dgsw;

namespace {

constexpr int kBlock = RED_BLOCK;                                  // elements per partial
constexpr int kMaxPartials = DGSW_L2_STATIC_MAX_ELEMS / kBlock;    // 4096
constexpr int kResultSlot = kMaxPartials;
constexpr int kMaxDevices = 64;
static_assert(DGSW_L2_STATIC_MAX_ELEMS % RED_BLOCK == 0, "limit must be whole blocks");

// the scratch: 4097 doubles (32 KiB + 8 B) per device
static __device__ __align__(256) double g_l2_scratch[kMaxPartials + 1];
// the degree-20 rule and the basis at its points, read uniformly by a warp: constant memory
static __constant__ L2Rule c_l2_rule;

struct FnParams {
    double v[DGSW_FN_PARAMS];
};

std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

template <int ND>
__global__ void __launch_bounds__(kBlock)
    l2_static_partials(const double* __restrict__ q, const int32_t* __restrict__ elem_nodes,
                       const double* __restrict__ node_xyz, int ne, int fn_set, FnParams fp, double t,
                       double* __restrict__ scratch) {
    __shared__ double sh[kBlock];
    const int e = blockIdx.x * kBlock + threadIdx.x;
    double val = 0.0;
    if (e < ne) {
        const int n0 = elem_nodes[3 * (size_t)e], n1 = elem_nodes[3 * (size_t)e + 1], n2 = elem_nodes[3 * (size_t)e + 2];
        const double x0 = node_xyz[3 * (size_t)n0], y0 = node_xyz[3 * (size_t)n0 + 1];
        const double x1 = node_xyz[3 * (size_t)n1], y1 = node_xyz[3 * (size_t)n1 + 1];
        const double x2 = node_xyz[3 * (size_t)n2], y2 = node_xyz[3 * (size_t)n2 + 1];
        const double J00 = (x1 - x0) / 2.0, J01 = (x2 - x0) / 2.0;
        const double J10 = (y1 - y0) / 2.0, J11 = (y2 - y0) / 2.0;
        const double aJ = fabs(J00 * J11 - J10 * J01);
        double qe[3][ND];
#pragma unroll
        for (int c = 0; c < 3 * ND; ++c) qe[c / ND][c % ND] = q[(size_t)e * 3 * ND + c];
        const double* phi = c_l2_rule.phi[ND == 3 ? 0 : 1];
        double l2[3] = {0.0, 0.0, 0.0};
        for (int gp = 0; gp < L2_NPT; ++gp) {
            const double x = x0 * c_l2_rule.psi[0][gp] + x1 * c_l2_rule.psi[1][gp] + x2 * c_l2_rule.psi[2][gp];
            const double y = y0 * c_l2_rule.psi[0][gp] + y1 * c_l2_rule.psi[1][gp] + y2 * c_l2_rule.psi[2][gp];
            const dgsw_fn3 f = dgsw_fn_true(fn_set, fp.v, t, x, y);
            const double tv[3] = {f.ze, f.qx, f.qy};
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                double u = 0.0;
#pragma unroll
                for (int k = 0; k < ND; ++k) u += qe[v][k] * phi[k * L2_NPT + gp];
                const double dd = tv[v] - u;
                l2[v] += (dd * dd) * c_l2_rule.w[gp];
            }
        }
        val = l2[0] * aJ + l2[1] * aJ + l2[2] * aJ;
    }
    const double s = block_sum(val, sh);
    if (threadIdx.x == 0) scratch[blockIdx.x] = s;
}

// one block: thread i adds partials i, i + 256, ... in order, then a fixed tree; deterministic
__global__ void __launch_bounds__(kBlock) l2_static_finish(double* __restrict__ scratch, int npartial) {
    __shared__ double sh[kBlock];
    double s = 0.0;
    for (int i = threadIdx.x; i < npartial; i += kBlock) s += scratch[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) scratch[kResultSlot] = s;
}

// once per device, with that device current: fill the rule and look up the scratch address. The result is
// kept for the life of the process: after a cudaDeviceReset the saved address and the constant-memory rule
// would be stale, so a reset between calls is not supported.
int setup_device(int dev, double** out, std::string& err) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev]) {
        *out = g_scratch_ptr[dev];
        return DGSW_OK;
    }
    static L2Rule rule;  // host copy, built once (guarded by the mutex)
    static bool rule_ready = false;
    if (!rule_ready) {
        Rule2D r = triangle_rule(20);
        if ((int)r.w.size() != L2_NPT) {
            err = "unexpected L2 rule size";
            return DGSW_ERR_UNSUPPORTED;
        }
        std::memset(&rule, 0, sizeof(rule));
        for (int i = 0; i < L2_NPT; ++i) {
            rule.w[i] = r.w[i];
            rule.psi[0][i] = -(r.z1[i] + r.z2[i]) / 2;
            rule.psi[1][i] = (1 + r.z1[i]) / 2;
            rule.psi[2][i] = (1 + r.z2[i]) / 2;
        }
        eval_basis(1, r.z1.data(), r.z2.data(), L2_NPT, rule.phi[0]);
        eval_basis(2, r.z1.data(), r.z2.data(), L2_NPT, rule.phi[1]);
        rule_ready = true;
    }
    cudaError_t e = cudaMemcpyToSymbol(c_l2_rule, &rule, sizeof(L2Rule));
    if (e != cudaSuccess) {
        err = std::string("cudaMemcpyToSymbol(L2 rule): ") + cudaGetErrorString(e);
        return DGSW_ERR_CUDA;
    }
    double* ptr = nullptr;
    e = cudaGetSymbolAddress((void**)&ptr, g_l2_scratch);
    if (e != cudaSuccess || !ptr) {
        err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
        return DGSW_ERR_CUDA;
    }
    g_scratch_ptr[dev] = ptr;
    *out = ptr;
    return DGSW_OK;
}

}  // namespace

namespace dgsw {
int set_last_error(int code, const std::string& msg);  // api.cu
}

extern "C" int32_t dgsw_l2_error_static(int32_t p, int64_t n_elems, const double* d_q, const int32_t* d_elem_nodes,
                                        const double* d_node_xyz, int32_t function_set, const double* fn_params,
                                        double t, void* stream, double* out) {
    if (!d_q || !d_elem_nodes || !d_node_xyz || !out)
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_l2_error_static: null argument");
    if (p != 1 && p != 2)
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_l2_error_static: p must be 1 or 2");
    if (n_elems <= 0 || n_elems > DGSW_L2_STATIC_MAX_ELEMS)
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT,
                                    "dgsw_l2_error_static: n_elems = " + std::to_string((long long)n_elems) +
                                        " is outside 1.." + std::to_string(DGSW_L2_STATIC_MAX_ELEMS) +
                                        " (the size of its static scratch); use dgsw_rkdg_l2_error for larger meshes");
    if (function_set < 0 || function_set >= DGSW_FN_COUNT)
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_l2_error_static: unknown function set");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return dgsw::set_last_error(DGSW_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return dgsw::set_last_error(DGSW_ERR_UNSUPPORTED, "dgsw_l2_error_static: device index beyond 63");
    double* scratch = nullptr;
    std::string err;
    int rc = setup_device(dev, &scratch, err);
    if (rc) return dgsw::set_last_error(rc, "dgsw_l2_error_static: " + err);

    FnParams fp;
    for (int i = 0; i < DGSW_FN_PARAMS; ++i) fp.v[i] = fn_params ? fn_params[i] : 0.0;
    const cudaStream_t st = (cudaStream_t)stream;
    const int ne = (int)n_elems;
    const int nblocks = (ne + kBlock - 1) / kBlock;  // <= kMaxPartials by the size check
    if (p == 1)
        l2_static_partials<3><<<nblocks, kBlock, 0, st>>>(d_q, d_elem_nodes, d_node_xyz, ne, function_set, fp, t, scratch);
    else
        l2_static_partials<6><<<nblocks, kBlock, 0, st>>>(d_q, d_elem_nodes, d_node_xyz, ne, function_set, fp, t, scratch);
    l2_static_finish<<<1, kBlock, 0, st>>>(scratch, nblocks);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return dgsw::set_last_error(DGSW_ERR_CUDA, std::string("dgsw_l2_error_static launch: ") + cudaGetErrorString(e));
    double s = 0.0;
    e = cudaMemcpyAsync(&s, scratch + kResultSlot, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return dgsw::set_last_error(DGSW_ERR_CUDA, std::string("dgsw_l2_error_static: ") + cudaGetErrorString(e));
    *out = std::sqrt(s);
    return DGSW_OK;
}
