// Launchers of the troubled-cell indicator kernels and the handle-free MLP entry points of the C ABI
// (dgsw_mlp_forward, dgsw_mlp_grad, dgsw_mlp_grad_work_floats, dgsw_mlp_adam).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/dgsw_rkdg.h"
#include "indicator.cuh"

namespace dgsw {

int set_last_error(int code, const std::string& msg);  // api.cu

namespace {
int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}
}  // namespace

// ------------------------------------------------------------------------------------------------
// FP32 CUDA-core forward and training kernels

__global__ void __launch_bounds__(128) mlp_forward_f32_kernel(const float* __restrict__ X, int64_t n,
                                                              const float* __restrict__ Pg, float* __restrict__ p) {
    __shared__ float Ps[MLP_NPARAM];
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) Ps[i] = Pg[i];
    __syncthreads();
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[MLP_IN], h1[MLP_H];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) x[k] = X[s * MLP_IN + k];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        float z = Ps[MLP_OFF_B1 + j];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) z = fmaf(Ps[MLP_OFF_W1 + j * MLP_IN + k], x[k], z);
        h1[j] = fmaxf(z, 0.0f);
    }
    float z3 = Ps[MLP_OFF_B3];
    for (int j = 0; j < MLP_H; ++j) {
        float z = Ps[MLP_OFF_B2 + j];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) z = fmaf(Ps[MLP_OFF_W2 + j * MLP_H + i], h1[i], z);
        z3 = fmaf(Ps[MLP_OFF_W3 + j], fmaxf(z, 0.0f), z3);
    }
    p[s] = sigmoidf_(z3);
}

// shared memory of mlp_grad_kernel (floats): parameters, then per-chunk inputs, activations and deltas
struct GradSmem {
    static constexpr int LD = MLP_H + 1;  // padded row of the [chunk][64] arrays
    static constexpr int P = 0;
    static constexpr int X = P + MLP_NPARAM;
    static constexpr int H1 = X + MLP_GRAD_CHUNK * MLP_IN;
    static constexpr int H2 = H1 + MLP_GRAD_CHUNK * LD;
    static constexpr int D2 = H2 + MLP_GRAD_CHUNK * LD;
    static constexpr int D1 = D2 + MLP_GRAD_CHUNK * LD;
    static constexpr int D3 = D1 + MLP_GRAD_CHUNK * LD;
    static constexpr int LOSS = D3 + MLP_GRAD_CHUNK;
    static constexpr int TOTAL = LOSS + MLP_GRAD_CHUNK;
    static constexpr size_t bytes() { return (size_t)TOTAL * sizeof(float); }
};
constexpr int MLP_GRAD_PER_THREAD = (MLP_NPARAM + MLP_GRAD_CHUNK - 1) / MLP_GRAD_CHUNK;  // 43

// Block b accumulates the unnormalised gradient of chunks b, b + gridDim.x, ... (chunk = 128 samples,
// one per thread) and writes partial[b][0..NPARAM) plus its loss sum to partial[b][NPARAM]. Thread t
// owns parameters t, t + 128, ...: each sum runs over the chunk's samples in order, so the result
// does not depend on scheduling.
__global__ void __launch_bounds__(MLP_GRAD_CHUNK) mlp_grad_kernel(const float* __restrict__ X,
                                                                  const uint8_t* __restrict__ y, int64_t n,
                                                                  const float* __restrict__ Pg, float pos_weight,
                                                                  float* __restrict__ partial) {
    extern __shared__ float gs[];
    using S = GradSmem;
    float* Ps = gs + S::P;
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) Ps[i] = Pg[i];
    float acc[MLP_GRAD_PER_THREAD];
#pragma unroll
    for (int r = 0; r < MLP_GRAD_PER_THREAD; ++r) acc[r] = 0.0f;
    float loss_acc = 0.0f;
    const int t = threadIdx.x;
    const int64_t nchunks = (n + MLP_GRAD_CHUNK - 1) / MLP_GRAD_CHUNK;
    for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        __syncthreads();
        const int64_t s = ch * MLP_GRAD_CHUNK + t;
        const bool valid = s < n;
        float* xs = gs + S::X + t * MLP_IN;
        float* h1 = gs + S::H1 + t * S::LD;
        float* h2 = gs + S::H2 + t * S::LD;
        float* d2 = gs + S::D2 + t * S::LD;
        float* d1 = gs + S::D1 + t * S::LD;
        float yv = 0.0f;
        if (valid) {
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) xs[k] = X[s * MLP_IN + k];
            yv = y[s] ? 1.0f : 0.0f;
        } else {
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) xs[k] = 0.0f;
        }
        // forward
        for (int j = 0; j < MLP_H; ++j) {
            float z = Ps[MLP_OFF_B1 + j];
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) z = fmaf(Ps[MLP_OFF_W1 + j * MLP_IN + k], xs[k], z);
            h1[j] = z;  // pre-activation kept for the ReLU mask
        }
        float z3 = Ps[MLP_OFF_B3];
        for (int j = 0; j < MLP_H; ++j) {
            float z = Ps[MLP_OFF_B2 + j];
            for (int i = 0; i < MLP_H; ++i) z = fmaf(Ps[MLP_OFF_W2 + j * MLP_H + i], fmaxf(h1[i], 0.0f), z);
            h2[j] = z;
            z3 = fmaf(Ps[MLP_OFF_W3 + j], fmaxf(z, 0.0f), z3);
        }
        const float p = sigmoidf_(z3);
        const float wy = pos_weight * yv;
        // loss: w y softplus(-z) + (1 - y) softplus(z)
        const float sp_pos = fmaxf(z3, 0.0f) + log1pf(expf(-fabsf(z3)));
        const float sp_neg = sp_pos - z3;
        const float d3 = valid ? p * (1.0f - yv) - wy * (1.0f - p) : 0.0f;
        gs[S::D3 + t] = d3;
        gs[S::LOSS + t] = valid ? wy * sp_neg + (1.0f - yv) * sp_pos : 0.0f;
        // backward through layer 2 and 1
        for (int j = 0; j < MLP_H; ++j) d2[j] = h2[j] > 0.0f ? d3 * Ps[MLP_OFF_W3 + j] : 0.0f;
        for (int i = 0; i < MLP_H; ++i) {
            float z = 0.0f;
            for (int j = 0; j < MLP_H; ++j) z = fmaf(Ps[MLP_OFF_W2 + j * MLP_H + i], d2[j], z);
            d1[i] = h1[i] > 0.0f ? z : 0.0f;
        }
        // activations for the weight gradients: h1 and h2 after the ReLU
        for (int j = 0; j < MLP_H; ++j) {
            h1[j] = fmaxf(h1[j], 0.0f);
            h2[j] = fmaxf(h2[j], 0.0f);
        }
        __syncthreads();
        if (t == 0)
            for (int i = 0; i < MLP_GRAD_CHUNK; ++i) loss_acc += gs[S::LOSS + i];
#pragma unroll
        for (int r = 0; r < MLP_GRAD_PER_THREAD; ++r) {
            const int q = t + r * MLP_GRAD_CHUNK;
            if (q >= MLP_NPARAM) break;
            float g = 0.0f;
            if (q < MLP_OFF_B1) {
                const int j = q / MLP_IN, k = q % MLP_IN;
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g = fmaf(gs[S::D1 + i * S::LD + j], gs[S::X + i * MLP_IN + k], g);
            } else if (q < MLP_OFF_W2) {
                const int j = q - MLP_OFF_B1;
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g += gs[S::D1 + i * S::LD + j];
            } else if (q < MLP_OFF_B2) {
                const int j = (q - MLP_OFF_W2) / MLP_H, k = (q - MLP_OFF_W2) % MLP_H;
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g = fmaf(gs[S::D2 + i * S::LD + j], gs[S::H1 + i * S::LD + k], g);
            } else if (q < MLP_OFF_W3) {
                const int j = q - MLP_OFF_B2;
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g += gs[S::D2 + i * S::LD + j];
            } else if (q < MLP_OFF_B3) {
                const int j = q - MLP_OFF_W3;
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g = fmaf(gs[S::D3 + i], gs[S::H2 + i * S::LD + j], g);
            } else {
                for (int i = 0; i < MLP_GRAD_CHUNK; ++i) g += gs[S::D3 + i];
            }
            acc[r] += g;
        }
    }
    float* out = partial + (size_t)blockIdx.x * (MLP_NPARAM + 1);
#pragma unroll
    for (int r = 0; r < MLP_GRAD_PER_THREAD; ++r) {
        const int q = t + r * MLP_GRAD_CHUNK;
        if (q < MLP_NPARAM) out[q] = acc[r];
    }
    if (t == 0) out[MLP_NPARAM] = loss_acc;
}

// grad[i] = sum_b partial[b][i] / n in block order; loss likewise (into loss_out[0], FP64)
__global__ void __launch_bounds__(256) mlp_grad_reduce_kernel(const float* __restrict__ partial, int nblocks,
                                                              int64_t n, float* __restrict__ grad,
                                                              double* __restrict__ loss_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > MLP_NPARAM) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += (double)partial[(size_t)b * (MLP_NPARAM + 1) + i];
    if (i < MLP_NPARAM)
        grad[i] = (float)(s / (double)n);
    else if (loss_out)
        loss_out[0] = s / (double)n;
}

// Adam (Kingma & Ba 2015) with the bias corrections c1 = 1 / (1 - beta1^t), c2 = 1 / (1 - beta2^t)
__global__ void __launch_bounds__(256) mlp_adam_kernel(float* __restrict__ P, float* __restrict__ m,
                                                       float* __restrict__ v, const float* __restrict__ g, int n,
                                                       float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

template <typename Real>
cudaError_t launch_indicator_features(const FeatureArgs<Real>& F, const int* ref_of_dev, float* feat, uint8_t* ok,
                                      cudaStream_t s) {
    if (F.ne <= 0) return cudaSuccess;
    indicator_features_kernel<Real><<<(F.ne + 255) / 256, 256, 0, s>>>(F, ref_of_dev, feat, ok);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_mlp_tc(const TcArgs& T, const FeatureArgs<Real>& F, cudaStream_t s) {
    const int64_t nrows = T.mode == 0 ? T.n : (int64_t)F.ne;
    if (nrows <= 0) return cudaSuccess;
    const int64_t ntiles = (nrows + MLP_TILE - 1) / MLP_TILE;
    static bool attr_set[2] = {false, false};
    const int which = sizeof(Real) == 4 ? 0 : 1;
    if (!attr_set[which]) {
        cudaError_t e = cudaFuncSetAttribute(mlp_tc_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             TcSmem::TOTAL + 1024);
        if (e != cudaSuccess) return e;
        attr_set[which] = true;
    }
    const int grid = (int)std::min<int64_t>(ntiles, (int64_t)sm_count() * MLP_TC_CTAS_PER_SM);
    mlp_tc_kernel<Real><<<grid, MLP_TILE, TcSmem::TOTAL + 1024, s>>>(T, F);
    return cudaGetLastError();
}

template cudaError_t launch_indicator_features<float>(const FeatureArgs<float>&, const int*, float*, uint8_t*,
                                                      cudaStream_t);
template cudaError_t launch_indicator_features<double>(const FeatureArgs<double>&, const int*, float*, uint8_t*,
                                                       cudaStream_t);
template cudaError_t launch_mlp_tc<float>(const TcArgs&, const FeatureArgs<float>&, cudaStream_t);
template cudaError_t launch_mlp_tc<double>(const TcArgs&, const FeatureArgs<double>&, cudaStream_t);

}  // namespace dgsw

using namespace dgsw;

namespace {
// error flag of the handle-free tensor-core forward (a wait that timed out); no allocation needed
__device__ int g_tc_error;

int grad_blocks(int64_t n) {
    const int64_t chunks = (n + MLP_GRAD_CHUNK - 1) / MLP_GRAD_CHUNK;
    return (int)std::max<int64_t>(1, std::min<int64_t>(chunks, 4 * 148));
}
}  // namespace

extern "C" {

int32_t dgsw_mlp_forward(const float* d_x, int64_t n, const float* d_params, float* d_p, int32_t tensor_cores,
                         void* stream) {
    if (!d_x || !d_params || !d_p || n < 0)
        return set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_mlp_forward: null pointer or negative n");
    if (n == 0) return DGSW_OK;
    if (n > ((int64_t)1 << 31) - MLP_TILE)
        return set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_mlp_forward: n beyond 2^31 rows");
    const cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (tensor_cores) {
        int* err = nullptr;
        e = cudaGetSymbolAddress((void**)&err, g_tc_error);
        if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
        TcArgs T{};
        T.params = d_params;
        T.X = d_x;
        T.p = d_p;
        T.n = n;
        T.mode = 0;
        T.error = err;
        FeatureArgs<float> F{};
        if (e == cudaSuccess) e = launch_mlp_tc<float>(T, F, s);
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && herr)
            return set_last_error(DGSW_ERR_CUDA, "dgsw_mlp_forward: tensor-core wait timed out");
    } else {
        mlp_forward_f32_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_x, n, d_params, d_p);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return set_last_error(DGSW_ERR_CUDA, std::string("dgsw_mlp_forward: ") + cudaGetErrorString(e));
    return DGSW_OK;
}

int64_t dgsw_mlp_grad_work_floats(int64_t n) { return (int64_t)grad_blocks(n) * (MLP_NPARAM + 1); }

int32_t dgsw_mlp_grad(const float* d_x, const uint8_t* d_y, int64_t n, const float* d_params, float pos_weight,
                      float* d_grad, float* d_work, int64_t work_floats, double* d_loss, void* stream) {
    if (!d_x || !d_y || !d_params || !d_grad || !d_work || n <= 0)
        return set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_mlp_grad: null pointer or empty batch");
    const int nb = grad_blocks(n);
    if (work_floats < (int64_t)nb * (MLP_NPARAM + 1))
        return set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_mlp_grad: work buffer smaller than "
                                                         "dgsw_mlp_grad_work_floats(n)");
    const cudaStream_t s = (cudaStream_t)stream;
    static bool attr = false;
    cudaError_t e = cudaSuccess;
    if (!attr) {
        e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GradSmem::bytes());
        attr = e == cudaSuccess;
    }
    if (e == cudaSuccess) {
        mlp_grad_kernel<<<nb, MLP_GRAD_CHUNK, GradSmem::bytes(), s>>>(d_x, d_y, n, d_params, pos_weight, d_work);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        mlp_grad_reduce_kernel<<<(MLP_NPARAM + 1 + 255) / 256, 256, 0, s>>>(d_work, nb, n, d_grad, d_loss);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return set_last_error(DGSW_ERR_CUDA, std::string("dgsw_mlp_grad: ") + cudaGetErrorString(e));
    return DGSW_OK;
}

int32_t dgsw_mlp_adam(float* d_params, float* d_m, float* d_v, const float* d_grad, int32_t step, float lr,
                      float beta1, float beta2, float eps, void* stream) {
    if (!d_params || !d_m || !d_v || !d_grad || step < 1)
        return set_last_error(DGSW_ERR_INVALID_ARGUMENT, "dgsw_mlp_adam: null pointer or step < 1");
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)beta1, step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)beta2, step)));
    mlp_adam_kernel<<<(MLP_NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_m, d_v, d_grad, MLP_NPARAM,
                                                                                lr, beta1, beta2, eps, c1, c2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_last_error(DGSW_ERR_CUDA, std::string("dgsw_mlp_adam: ") + cudaGetErrorString(e));
    return DGSW_OK;
}

}  // extern "C"
