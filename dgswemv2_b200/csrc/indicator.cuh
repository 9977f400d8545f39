// Learned troubled-cell indicator: an 18 -> 64 -> 64 -> 1 MLP (ReLU, sigmoid) that predicts the
// Cockburn-Shu limiter's own decision (CS_slope_limiter_serial, source/problem/SWE/problem_slope_limiter/
// swe_CS_slope_limiter.hpp:89-189: "this cell's state changes") from the quantities that limiter reads,
// and gates which cells the limiter pass visits. No counterpart in the reference.
//
// Kernels:
//   indicator_features_kernel  the 18 scale-free features of each element (FP64 arithmetic, FP32 out)
//   mlp_forward_f32_kernel     FP32 CUDA-core forward (training-time evaluation)
//   mlp_grad_kernel            per-block FP32 gradient partials of the weighted BCE loss (fixed order)
//   mlp_grad_reduce_kernel     partials -> mean gradient and loss, in block order (deterministic)
//   mlp_adam_kernel            Adam on the FP32 master parameters
//   mlp_tc_kernel              inference on the tensor cores: features -> BF16 tile in shared memory,
//                              two tcgen05.mma GEMMs with FP32 accumulators in TMEM, ReLU/sigmoid
//                              epilogues from tcgen05.ld; optionally the gate (limiter work list)
// Parameter vector (FP32, 5441 values): W1[64][18], b1[64], W2[64][64], b2[64], w3[64], b3.
#ifndef DGSW_INDICATOR_CUH
#define DGSW_INDICATOR_CUH

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcgen05.cuh"

namespace dgsw {

constexpr int MLP_IN = 18, MLP_H = 64;
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B3 + 1;  // 5441
constexpr int MLP_TILE = 128;               // rows per tensor-core tile (MMA M)
constexpr int MLP_K1 = 32;                  // first-layer K, 18 features zero-padded
constexpr int MLP_GRAD_CHUNK = 128;         // samples per gradient chunk (one per thread)

// indicator statistics counters (unsigned long long each)
enum { IND_CONSIDERED = 0, IND_LISTED = 1, IND_LIMITED = 2, IND_MISSED = 3, IND_COUNT = 4, IND_NCOUNTERS = 5 };

template <typename Real>
struct FeatureArgs {
    const Real* q;             // [(var*ND+dof)][ne_pad], device order
    const unsigned char* wet;  // wet flags of this state
    const int* nbr;            // [3][ne_pad]: neighbour device index, or -2 - boundary type
    const int* enodes;         // [3][ne_pad]
    const double2* xy;         // node coordinates
    const double* nz;          // node depths
    int ne, ne_pad, nd;
    double g, M;               // gravity, TVB constant of the limiter
    int fset;                  // feature set: 0 characteristic (below), 1 the raw modal coefficients and
                               // neighbour cell means
};

constexpr int IND_FEATURES_CHARACTERISTIC = 0, IND_FEATURES_RAW = 1;

// The 18 features of element e and whether the limiter looks at the cell (it and its neighbours wet,
// boundary faces land or function). Feature set 0 (definition in oracle/mlp_oracle.py): fields in
// characteristic units, one common scale, TVB ratio, Froude numbers. Feature set 1, the literal input list
// of the learned-indicator workload: the p = 1 modal coefficients of ze, qx, qy (3 x 3) and the cell means
// of the three neighbours of each field (9; a boundary face repeats the cell's own mean). FP64 arithmetic
// with explicit roundings (no contraction), so the host oracle reproduces the values bit for bit.
template <typename Real>
__device__ __forceinline__ bool element_features(const FeatureArgs<Real>& F, int e, float* out) {
    const size_t P = (size_t)F.ne_pad;
    const int ND = F.nd;
    double a[3], b[3], c[3], d[3][3];
    bool ok = F.wet[e] != 0;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        a[v] = (double)F.q[(size_t)(v * ND) * P + e];
        b[v] = (double)F.q[(size_t)(v * ND + 1) * P + e];
        c[v] = (double)F.q[(size_t)(v * ND + 2) * P + e];
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const int m = F.nbr[f * P + e];
        if (m >= 0) {
            ok = ok && (F.wet[m] != 0);
#pragma unroll
            for (int v = 0; v < 3; ++v) d[f][v] = __dsub_rn((double)F.q[(size_t)(v * ND) * P + m], a[v]);
            if (F.fset == IND_FEATURES_RAW) {
#pragma unroll
                for (int v = 0; v < 3; ++v) out[9 + 3 * f + v] = __double2float_rn((double)F.q[(size_t)(v * ND) * P + m]);
            }
        } else {
            const int bt = -2 - m;
            // land, tide, flow and function boundaries: wet_neigh is the element's own flag
            ok = ok && (bt >= 0 && bt <= 3);
#pragma unroll
            for (int v = 0; v < 3; ++v) d[f][v] = 0.0;
            if (F.fset == IND_FEATURES_RAW) {
#pragma unroll
                for (int v = 0; v < 3; ++v) out[9 + 3 * f + v] = __double2float_rn(a[v]);
            }
        }
    }
    if (F.fset == IND_FEATURES_RAW) {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            out[3 * v] = __double2float_rn(a[v]);
            out[3 * v + 1] = __double2float_rn(b[v]);
            out[3 * v + 2] = __double2float_rn(c[v]);
        }
        return ok;
    }
    const int n[3] = {F.enodes[e], F.enodes[P + e], F.enodes[2 * P + e]};
    const double third = 1.0 / 3.0;
    const double zb = __dadd_rn(__dadd_rn(__dmul_rn(F.nz[n[0]], third), __dmul_rn(F.nz[n[1]], third)),
                                __dmul_rn(F.nz[n[2]], third));
    const double H = fmax(__dadd_rn(a[0], zb), 1.0e-3);
    const double ic = __ddiv_rn(1.0, __dsqrt_rn(__dmul_rn(F.g, H)));
#pragma unroll
    for (int v = 1; v < 3; ++v) {
        b[v] = __dmul_rn(b[v], ic);
        c[v] = __dmul_rn(c[v], ic);
#pragma unroll
        for (int f = 0; f < 3; ++f) d[f][v] = __dmul_rn(d[f][v], ic);
    }
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        s = fmax(s, fmax(fabs(b[v]), fabs(c[v])));
#pragma unroll
        for (int f = 0; f < 3; ++f) s = fmax(s, fabs(d[f][v]));
    }
    if (s == 0.0) s = 1.0;
    // mean squared distance from the centroid to the edge midpoints
    double X[3], Y[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double2 p = F.xy[n[k]];
        X[k] = p.x;
        Y[k] = p.y;
    }
    const double cx = __ddiv_rn(__dadd_rn(__dadd_rn(X[0], X[1]), X[2]), 3.0);
    const double cy = __ddiv_rn(__dadd_rn(__dadd_rn(Y[0], Y[1]), Y[2]), 3.0);
    double r2 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double mx = __dsub_rn(__ddiv_rn(__dadd_rn(X[(k + 1) % 3], X[(k + 2) % 3]), 2.0), cx);
        const double my = __dsub_rn(__ddiv_rn(__dadd_rn(Y[(k + 1) % 3], Y[(k + 2) % 3]), 2.0), cy);
        r2 = __dadd_rn(r2, __dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)));
    }
    r2 = __ddiv_rn(r2, 3.0);
    const double inv = __ddiv_rn(1.0, s);
    out[0] = __double2float_rn(__ddiv_rn(s, __dadd_rn(s, __dmul_rn(F.M, r2))));
    out[1] = __double2float_rn(fmin(fmax(__dmul_rn(__ddiv_rn(a[1], H), ic), -8.0), 8.0));
    out[2] = __double2float_rn(fmin(fmax(__dmul_rn(__ddiv_rn(a[2], H), ic), -8.0), 8.0));
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        out[3 + 5 * v] = __double2float_rn(__dmul_rn(b[v], inv));
        out[4 + 5 * v] = __double2float_rn(__dmul_rn(c[v], inv));
#pragma unroll
        for (int f = 0; f < 3; ++f) out[5 + 5 * v + f] = __double2float_rn(__dmul_rn(d[f][v], inv));
    }
    return ok;
}

// features of every element, written in reference order (row ref_of_dev[d] for device element d)
template <typename Real>
__global__ void __launch_bounds__(256) indicator_features_kernel(const FeatureArgs<Real> F, const int* ref_of_dev,
                                                                 float* __restrict__ feat, uint8_t* __restrict__ ok) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= F.ne) return;
    float x[MLP_IN];
    const bool k = element_features(F, d, x);
    const size_t r = (size_t)ref_of_dev[d];
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) feat[r * MLP_IN + i] = x[i];
    if (ok) ok[r] = k ? 1 : 0;
}

// ------------------------------------------------------------------------------------------------
// FP32 CUDA-core forward and training kernels

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

// ------------------------------------------------------------------------------------------------
// tensor-core inference

// shared memory of mlp_tc_kernel (bytes, 1024-aligned base)
struct TcSmem {
    // A1 and A2 share their space: A2 is written only after the layer-1 MMA has read A1, and the next
    // tile's A1 only after the layer-2 MMA has read A2
    static constexpr int A1 = 0;                                  // [128][32] BF16 features
    static constexpr int A2 = 0;                                  // [128][64] BF16 hidden layer 1
    static constexpr int B1 = A2 + MLP_TILE * MLP_H * 2;          // [64][32] BF16 W1 (K padded)
    static constexpr int B2 = B1 + MLP_H * MLP_K1 * 2;            // [64][64] BF16 W2
    static constexpr int VEC = B2 + MLP_H * MLP_H * 2;            // b1, b2, w3, b3 (FP32)
    static constexpr int BAR = VEC + 1024;                        // mbarrier, TMEM address
    static constexpr int TOTAL = BAR + 64;
};
constexpr int MLP_TMEM_COLS = 64;  // one 128 x 64 FP32 accumulator, reused by both layers
constexpr int MLP_TC_CTAS_PER_SM = 5;  // 5 x 64 TMEM columns <= 512; about 30 KB shared memory each

struct TcArgs {
    const float* params;  // FP32 master parameters
    // matrix input (mode 0): X [n][18] -> p [n]
    const float* X;
    float* p;
    int64_t n;
    // gate (mode 1: work list, mode 2: flags for the shadow limiter pass)
    int mode;
    float skip_below;          // p < skip_below: the limiter skips the cell
    int* list;                 // cells sent to the limiter (mode 1)
    int* list_count;
    unsigned char* gate;       // per cell: 1 if sent to the limiter
    unsigned char* limited;    // cleared for the cells the limiter will not visit
    unsigned long long* counters;
    int* error;                // set to 1 if a tensor-core wait timed out
};

// eight FP32 values -> eight BF16 (round to nearest even) in one 16-byte shared-memory store
__device__ __forceinline__ void store_bf16x8(__nv_bfloat16* dst, const float* v) {
    uint4 u;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t*>(&h0);
    u.y = *reinterpret_cast<uint32_t*>(&h1);
    u.z = *reinterpret_cast<uint32_t*>(&h2);
    u.w = *reinterpret_cast<uint32_t*>(&h3);
    *reinterpret_cast<uint4*>(dst) = u;
}

template <typename Real>
__global__ void __launch_bounds__(MLP_TILE, MLP_TC_CTAS_PER_SM) mlp_tc_kernel(const TcArgs T, const FeatureArgs<Real> F) {
    extern __shared__ __align__(1024) unsigned char tsm[];
    __nv_bfloat16* A1 = reinterpret_cast<__nv_bfloat16*>(tsm + TcSmem::A1);
    __nv_bfloat16* A2 = reinterpret_cast<__nv_bfloat16*>(tsm + TcSmem::A2);
    __nv_bfloat16* B1 = reinterpret_cast<__nv_bfloat16*>(tsm + TcSmem::B1);
    __nv_bfloat16* B2 = reinterpret_cast<__nv_bfloat16*>(tsm + TcSmem::B2);
    float* vb1 = reinterpret_cast<float*>(tsm + TcSmem::VEC);
    float* vb2 = vb1 + MLP_H;
    float* vw3 = vb2 + MLP_H;
    float* vb3 = vw3 + MLP_H;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + TcSmem::BAR);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tsm + TcSmem::BAR + 8);
    int* abort_flag = reinterpret_cast<int*>(tsm + TcSmem::BAR + 16);

    const int t = threadIdx.x, warp = t >> 5;
    // weights -> BF16 core-matrix tiles (W1 zero-padded from 18 to 32 columns)
    for (int i = t; i < MLP_H * MLP_K1; i += MLP_TILE) {
        const int j = i / MLP_K1, k = i % MLP_K1;
        const float w = k < MLP_IN ? T.params[MLP_OFF_W1 + j * MLP_IN + k] : 0.0f;
        B1[tc::cm_index(j, k, MLP_K1)] = __float2bfloat16_rn(w);
    }
    for (int i = t; i < MLP_H * MLP_H; i += MLP_TILE) {
        const int j = i / MLP_H, k = i % MLP_H;
        B2[tc::cm_index(j, k, MLP_H)] = __float2bfloat16_rn(T.params[MLP_OFF_W2 + i]);
    }
    if (t < MLP_H) {
        vb1[t] = T.params[MLP_OFF_B1 + t];
        vb2[t] = T.params[MLP_OFF_B2 + t];
        vw3[t] = T.params[MLP_OFF_W3 + t];
    }
    if (t == 0) {
        vb3[0] = T.params[MLP_OFF_B3];
        *abort_flag = 0;
        tc::mbar_init(mbar, 1);
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, MLP_TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t idesc = tc::idesc_bf16_f32(MLP_TILE, MLP_H);
    const uint32_t sA1 = tc::smem_u32(A1), sA2 = tc::smem_u32(A2), sB1 = tc::smem_u32(B1), sB2 = tc::smem_u32(B2);
    uint32_t phase = 0;
    const int64_t nrows = T.mode == 0 ? T.n : (int64_t)F.ne;
    const int64_t ntiles = (nrows + MLP_TILE - 1) / MLP_TILE;
    constexpr uint32_t kMaxPolls = 1u << 24;

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * MLP_TILE + t;
        const bool valid = row < nrows;
        float x[MLP_IN];
        bool ok = false;
        if (valid) {
            if (T.mode == 0) {
#pragma unroll
                for (int k = 0; k < MLP_IN; ++k) x[k] = T.X[row * MLP_IN + k];
                ok = true;
            } else {
                ok = element_features(F, (int)row, x);
            }
        } else {
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) x[k] = 0.0f;
        }
        // row t of the tile: four 16-byte core-matrix rows of 8 BF16 values
#pragma unroll
        for (int g = 0; g < MLP_K1 / 8; ++g) {
            float v8[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v8[i] = (g * 8 + i) < MLP_IN ? x[g * 8 + i] : 0.0f;
            store_bf16x8(A1 + tc::cm_index(t, g * 8, MLP_K1), v8);
        }
        tc::fence_proxy_async();
        __syncthreads();
        // layer 1: [128 x 32] x [32 x 64]
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < MLP_K1 / 16; ++kk)
                tc::mma_bf16(tmem, tc::smem_desc(sA1 + kk * 256, 128, (MLP_K1 / 8) * 128),
                             tc::smem_desc(sB1 + kk * 256, 128, (MLP_K1 / 8) * 128), idesc, kk > 0);
            tc::mma_commit(mbar);
        }
        if (!tc::mbar_wait_bounded(mbar, phase, kMaxPolls)) *abort_flag = 1;
        phase ^= 1;
        tc::fence_after_sync();
        __syncthreads();
        if (*abort_flag) break;
#pragma unroll
        for (int c = 0; c < MLP_H / 16; ++c) {
            float v[16];
            tc::tmem_ld16(lane_addr + c * 16, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + vb1[c * 16 + i], 0.0f);
            store_bf16x8(A2 + tc::cm_index(t, c * 16, MLP_H), v);
            store_bf16x8(A2 + tc::cm_index(t, c * 16 + 8, MLP_H), v + 8);
        }
        tc::fence_before_sync();
        tc::fence_proxy_async();
        __syncthreads();
        // layer 2: [128 x 64] x [64 x 64], into the same TMEM columns
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < MLP_H / 16; ++kk)
                tc::mma_bf16(tmem, tc::smem_desc(sA2 + kk * 256, 128, (MLP_H / 8) * 128),
                             tc::smem_desc(sB2 + kk * 256, 128, (MLP_H / 8) * 128), idesc, kk > 0);
            tc::mma_commit(mbar);
        }
        if (!tc::mbar_wait_bounded(mbar, phase, kMaxPolls)) *abort_flag = 1;
        phase ^= 1;
        tc::fence_after_sync();
        __syncthreads();
        if (*abort_flag) break;
        float z3 = vb3[0];
#pragma unroll
        for (int c = 0; c < MLP_H / 16; ++c) {
            float v[16];
            tc::tmem_ld16(lane_addr + c * 16, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) z3 = fmaf(vw3[c * 16 + i], fmaxf(v[i] + vb2[c * 16 + i], 0.0f), z3);
        }
        const float p = sigmoidf_(z3);
        if (T.mode == 0) {
            if (valid) T.p[row] = p;
        } else {
            // T.mode is uniform over the grid: the whole warp takes this branch
            const bool okc = valid && ok;
            const bool send = okc && p >= T.skip_below;
            if (valid) {
                if (T.p) T.p[row] = p;
                if (T.mode == 1) {
                    if (!send) T.limited[row] = 0;
                } else {
                    T.gate[row] = send ? 1 : 0;
                }
            }
            // warp-aggregated list append and counters
            const unsigned m_send = __ballot_sync(0xffffffffu, send);
            const unsigned m_ok = __ballot_sync(0xffffffffu, okc);
            const int lane = t & 31;
            int base = 0;
            if (T.mode == 1 && lane == 0 && m_send) base = atomicAdd(T.list_count, __popc(m_send));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (T.mode == 1 && send) T.list[base + __popc(m_send & ((1u << lane) - 1u))] = (int)row;
            if (lane == 0) {
                if (m_ok) atomicAdd(&T.counters[IND_CONSIDERED], (unsigned long long)__popc(m_ok));
                if (m_send) atomicAdd(&T.counters[IND_LISTED], (unsigned long long)__popc(m_send));
            }
        }
        // every thread's TMEM reads finish before the next tile's MMA overwrites the columns
        tc::fence_before_sync();
        __syncthreads();
    }
    if (*abort_flag && t == 0) atomicExch(T.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, MLP_TMEM_COLS);
}

// host launchers (indicator.cu)
template <typename Real>
cudaError_t launch_indicator_features(const FeatureArgs<Real>& F, const int* ref_of_dev, float* feat, uint8_t* ok,
                                      cudaStream_t s);
template <typename Real>
cudaError_t launch_mlp_tc(const TcArgs& T, const FeatureArgs<Real>& F, cudaStream_t s);

}  // namespace dgsw

#endif
