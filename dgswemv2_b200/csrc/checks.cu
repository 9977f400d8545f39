// Kernel self-checks: the stage kernel's own device functions (llf_flux, the ISP::Internal wet/dry
// fix-ups, wetting_drying from stage_kernel.cuh) run by small kernels on caller data, so that the
// reference's known-answer vectors (test/test_llf_flux.cpp, test/test_wetting_drying.cpp) and the oracle
// can be checked against the CUDA code itself rather than only through whole runs.
// Host arrays in and out; device buffers are allocated per call (these are test entry points).
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/dgsw_rkdg.h"
#include "stage_kernel.cuh"

namespace dgsw {
int set_last_error(int code, const std::string& msg);
}

namespace {

using dgsw::Flux2;

// the interface Gauss point of the stage kernel's phase 2 for an internal edge: LLF with sp on the in
// side, F_ex = -F_in, and the wet/dry fix-ups when either side is dry (rkdg_swe_is_internal.hpp:26-95)
template <typename Real>
__global__ void check_flux_kernel(int n, Real g, const double* __restrict__ qin, const double* __restrict__ qex,
                                  const double* __restrict__ bin, const double* __restrict__ bex,
                                  const double* __restrict__ sp, const double* __restrict__ nrm,
                                  const unsigned char* __restrict__ wet_in, const unsigned char* __restrict__ wet_ex,
                                  int internal, double* __restrict__ Fin, double* __restrict__ Fex) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Real qi[3] = {(Real)qin[3 * i], (Real)qin[3 * i + 1], (Real)qin[3 * i + 2]};
    const Real qe[3] = {(Real)qex[3 * i], (Real)qex[3 * i + 1], (Real)qex[3 * i + 2]};
    const Real nx = (Real)nrm[2 * i], ny = (Real)nrm[2 * i + 1];
    Real F[3];
    dgsw::llf_flux<Real>(g, qi, qe, (Real)bin[i], (Real)sp[i], nx, ny, F);
    Real E[3] = {-F[0], -F[1], -F[2]};
    if (internal) {
        const bool wa = wet_in[i] != 0, wb = wet_ex[i] != 0;
        if (!(wa && wb)) {
            const Flux2<Real> r = dgsw::wd_fixup<Real>(g, qi[0], qi[1], qi[2], qe[0], qe[1], qe[2], (Real)bin[i],
                                                       (Real)bex[i], (Real)sp[i], nx, ny, wa, wb, F[0], F[1], F[2]);
            F[0] = r.i0, F[1] = r.i1, F[2] = r.i2;
            E[0] = r.e0, E[1] = r.e1, E[2] = r.e2;
        }
    }
    for (int v = 0; v < 3; ++v) {
        Fin[3 * i + v] = (double)F[v];
        if (Fex) Fex[3 * i + v] = (double)E[v];
    }
}

// the stage kernel's wetting/drying pass (FP64 in both precisions) on p = 1 modal states
__global__ void check_wet_dry_kernel(int n, const double* __restrict__ q, const double* __restrict__ bv, double h_o,
                                     double thr, const unsigned char* __restrict__ wet_in, double* __restrict__ qo,
                                     unsigned char* __restrict__ wet_out, unsigned char* __restrict__ went_dry) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double qv[3][3];
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) qv[v][k] = q[9 * i + 3 * v + k];
    const double b[3] = {bv[3 * i], bv[3 * i + 1], bv[3 * i + 2]};
    const double bmin = fmin(b[0], fmin(b[1], b[2]));
    bool wd = false;
    const bool w = dgsw::wetting_drying<3, double>(qv, b, bmin, h_o, thr, wet_in[i] != 0, wd);
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) qo[9 * i + 3 * v + k] = qv[v][k];
    wet_out[i] = w ? 1 : 0;
    went_dry[i] = wd ? 1 : 0;
}

// device copies of host arrays, released at scope exit
struct Scratch {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T* in(const T* h, size_t n) {
        if (err != cudaSuccess || !h) return nullptr;
        void* d = nullptr;
        if ((err = cudaMalloc(&d, n * sizeof(T) + 16)) != cudaSuccess) return nullptr;
        ptrs.push_back(d);
        err = cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
        return (T*)d;
    }
    template <typename T>
    T* out(size_t n) {
        if (err != cudaSuccess) return nullptr;
        void* d = nullptr;
        if ((err = cudaMalloc(&d, n * sizeof(T) + 16)) != cudaSuccess) return nullptr;
        ptrs.push_back(d);
        return (T*)d;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
};

int cuda_fail(const char* what, cudaError_t e) {
    return dgsw::set_last_error(DGSW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return dgsw::set_last_error(DGSW_ERR_NO_DEVICE, "no CUDA device");
    }
    return DGSW_OK;
}

int run_flux(int32_t precision, int64_t n, double g, const double* q_in, const double* q_ex, const double* b_in,
             const double* b_ex, const double* sp, const double* normal, const uint8_t* wet_in, const uint8_t* wet_ex,
             int internal, double* F_in, double* F_ex) {
    if (n <= 0 || n > (1 << 24) || !q_in || !q_ex || !b_in || !sp || !normal || !F_in ||
        (internal && (!b_ex || !wet_in || !wet_ex)) || (precision != DGSW_FP64 && precision != DGSW_FP32))
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "flux check: bad arguments");
    if (int rc = check_device()) return rc;
    Scratch S;
    const size_t m = (size_t)n;
    const double *dqi = S.in(q_in, 3 * m), *dqe = S.in(q_ex, 3 * m), *dbi = S.in(b_in, m);
    const double* dbe = internal ? S.in(b_ex, m) : dbi;
    const double *dsp = S.in(sp, m), *dn = S.in(normal, 2 * m);
    const unsigned char* dwi = internal ? S.in(wet_in, m) : nullptr;
    const unsigned char* dwe = internal ? S.in(wet_ex, m) : nullptr;
    double* dFi = S.out<double>(3 * m);
    double* dFe = F_ex ? S.out<double>(3 * m) : nullptr;
    if (S.err != cudaSuccess) return cuda_fail("flux check", S.err);
    const unsigned blocks = (unsigned)((n + 127) / 128);
    if (precision == DGSW_FP64)
        check_flux_kernel<double><<<blocks, 128>>>((int)n, g, dqi, dqe, dbi, dbe, dsp, dn, dwi, dwe, internal, dFi, dFe);
    else
        check_flux_kernel<float><<<blocks, 128>>>((int)n, (float)g, dqi, dqe, dbi, dbe, dsp, dn, dwi, dwe, internal, dFi,
                                                  dFe);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(F_in, dFi, 3 * m * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && F_ex) e = cudaMemcpy(F_ex, dFe, 3 * m * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail("flux check", e);
    return DGSW_OK;
}

}  // namespace

extern "C" {

int32_t dgsw_check_llf_flux(int32_t precision, int64_t n, double g, const double* q_in, const double* q_ex,
                            const double* bath, const double* sp, const double* normal, double* F) {
    return run_flux(precision, n, g, q_in, q_ex, bath, nullptr, sp, normal, nullptr, nullptr, 0, F, nullptr);
}

int32_t dgsw_check_internal_flux(int32_t precision, int64_t n, double g, const double* q_in, const double* q_ex,
                                 const double* bath_in, const double* bath_ex, const double* sp, const double* normal,
                                 const uint8_t* wet_in, const uint8_t* wet_ex, double* F_in, double* F_ex) {
    if (!F_ex) return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "flux check: F_ex is required");
    return run_flux(precision, n, g, q_in, q_ex, bath_in, bath_ex, sp, normal, wet_in, wet_ex, 1, F_in, F_ex);
}

int32_t dgsw_check_wetting_drying(int64_t n, const double* q, const double* bath_vrtx, double h_o,
                                  const uint8_t* wet_in, double* q_out, uint8_t* wet_out, uint8_t* went_dry) {
    if (n <= 0 || n > (1 << 24) || !q || !bath_vrtx || !wet_in || !q_out || !wet_out || !(h_o > 0.0))
        return dgsw::set_last_error(DGSW_ERR_INVALID_ARGUMENT, "wetting/drying check: bad arguments");
    if (int rc = check_device()) return rc;
    Scratch S;
    const size_t m = (size_t)n;
    const double *dq = S.in(q, 9 * m), *db = S.in(bath_vrtx, 3 * m);
    const unsigned char* dw = S.in(wet_in, m);
    double* dqo = S.out<double>(9 * m);
    unsigned char *dwo = S.out<unsigned char>(m), *dwd = S.out<unsigned char>(m);
    if (S.err != cudaSuccess) return cuda_fail("wetting/drying check", S.err);
    // the threshold of swe_pre_init_prob_params.hpp:36, as the library sets it for a handle
    const double thr = 1.0e6 * h_o * 2.220446049250313e-16;
    check_wet_dry_kernel<<<(unsigned)((n + 127) / 128), 128>>>((int)n, dq, db, h_o, thr, dw, dqo, dwo, dwd);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(q_out, dqo, 9 * m * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(wet_out, dwo, m, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && went_dry) e = cudaMemcpy(went_dry, dwd, m, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail("wetting/drying check", e);
    return DGSW_OK;
}

}  // extern "C"
