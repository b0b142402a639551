// router.cu -- training and inference kernels of the learned precision router
// (router.cuh has the network and the features).  Inference is
// mlp_forward_tc_kernel, the arithmetic the routing pass runs (FP16 tensor-
// core products); mlp_forward_kernel is the FP32 forward of training.
//
// Training is mini-batch Adam on the mean squared error of the predicted
// log10 deposit.  A step is three kernels, all FP32 and deterministic:
//   mlp_fwd_bwd_kernel    one thread per sample: forward, loss, and the
//                         per-sample backward quantities (h1, h2, da1, da2,
//                         dy) into a scratch buffer;
//   mlp_grad_kernel       one thread per trainable parameter: the batch sum
//                         of its gradient, in sample order (no atomics);
//   mlp_adam_kernel       the Adam update (mu and sd are not trained).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/fjb.h"
#include "router.cuh"

namespace fjb {
namespace {

constexpr int kScratch = 4 * kHid + 1;  // h1, h2, da1, da2, dy per sample

__global__ void mlp_forward_kernel(const float *__restrict__ p, const float *__restrict__ X, int n,
                                   float *__restrict__ Y) {
    __shared__ float sp[kNParams];
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) sp[i] = p[i];
    __syncthreads();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float x[kFeat];
        for (int i = 0; i < kFeat; ++i) x[i] = X[(size_t)s * kFeat + i];
        Y[s] = mlp_forward(sp, x, nullptr, nullptr);
    }
}

// The router's inference arithmetic (mlp_forward_tc), a warp per 32 samples.
__global__ void mlp_forward_tc_kernel(const float *__restrict__ p, const float *__restrict__ X, int n,
                                      float *__restrict__ Y) {
    __shared__ float sp[kNParams];
    __shared__ __align__(16) __half wh[kTcSmemHalves];
    __shared__ __align__(16) __half xs[4][32 * kXRow];
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) sp[i] = p[i];
    stage_mlp_half(p, wh, wh + kHid * kW1Row);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warp = blockIdx.x * (blockDim.x >> 5) + w, nwarps = gridDim.x * (blockDim.x >> 5);
    for (int s0 = 32 * warp; s0 < n; s0 += 32 * nwarps) {  // warp-uniform
        const int s = s0 + lane;
        float x[kFeat];
        for (int i = 0; i < kFeat; ++i) x[i] = s < n ? X[(size_t)s * kFeat + i] : sp[kOffMu + i];
        const float y = mlp_forward_tc(sp, wh, wh + kHid * kW1Row, xs[w], x);
        if (s < n) Y[s] = y;
    }
}

__global__ void mlp_fwd_bwd_kernel(const float *__restrict__ p, const float *__restrict__ X,
                                   const float *__restrict__ T, int n, float *__restrict__ S,
                                   float *__restrict__ sq_err) {
    __shared__ float sp[kNParams];
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) sp[i] = p[i];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[kFeat], h1[kHid], h2[kHid];
    for (int i = 0; i < kFeat; ++i) x[i] = X[(size_t)s * kFeat + i];
    const float y = mlp_forward(sp, x, h1, h2);
    const float r = y - T[s];
    sq_err[s] = r * r;
    const float dy = 2.0f * r / (float)n;
    float *o = S + (size_t)s * kScratch;
    float da2[kHid];
    for (int k = 0; k < kHid; ++k) {
        da2[k] = dy * sp[kOffW3 + k] * (1.0f - h2[k] * h2[k]);
        o[kHid + k] = h2[k];
        o[3 * kHid + k] = da2[k];
    }
    for (int j = 0; j < kHid; ++j) {
        float dh = 0.0f;
        for (int k = 0; k < kHid; ++k) dh += da2[k] * sp[kOffW2 + k * kHid + j];
        o[j] = h1[j];
        o[2 * kHid + j] = dh * (1.0f - h1[j] * h1[j]);
    }
    o[4 * kHid] = dy;
}

__global__ void mlp_grad_kernel(const float *__restrict__ p, const float *__restrict__ X, int n,
                                const float *__restrict__ S, float *__restrict__ g) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < kOffW1 || q >= kNParams) return;
    float acc = 0.0f;
    if (q < kOffB1) {  // W1[j][i]: da1[j] * xn[i]
        const int j = (q - kOffW1) / kFeat, i = (q - kOffW1) % kFeat;
        const float mu = p[kOffMu + i], sd = p[kOffSd + i];
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 2 * kHid + j] * ((X[(size_t)s * kFeat + i] - mu) / sd);
    } else if (q < kOffW2) {  // b1[j]
        const int j = q - kOffB1;
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 2 * kHid + j];
    } else if (q < kOffB2) {  // W2[k][j]: da2[k] * h1[j]
        const int k = (q - kOffW2) / kHid, j = (q - kOffW2) % kHid;
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 3 * kHid + k] * S[(size_t)s * kScratch + j];
    } else if (q < kOffW3) {  // b2[k]
        const int k = q - kOffB2;
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 3 * kHid + k];
    } else if (q < kOffB3) {  // w3[k]: dy * h2[k]
        const int k = q - kOffW3;
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 4 * kHid] * S[(size_t)s * kScratch + kHid + k];
    } else {  // b3
        for (int s = 0; s < n; ++s) acc += S[(size_t)s * kScratch + 4 * kHid];
    }
    g[q] = acc;
}

__global__ void mlp_adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                                float *__restrict__ v, float lr, float b1, float b2, float eps, int step) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < kOffW1 || q >= kNParams) return;
    const float gq = g[q];
    m[q] = b1 * m[q] + (1.0f - b1) * gq;
    v[q] = b2 * v[q] + (1.0f - b2) * gq * gq;
    const float mh = m[q] / (1.0f - powf(b1, (float)step));
    const float vh = v[q] / (1.0f - powf(b2, (float)step));
    p[q] -= lr * mh / (sqrtf(vh) + eps);
}

thread_local std::string g_router_err;

int rfail(const char *msg, cudaError_t e = cudaSuccess) {
    g_router_err = std::string(msg) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return FJB_E_CUDA;
}

}  // namespace
}  // namespace fjb

using namespace fjb;

extern "C" {

int fjb_mlp_n_params(void) { return kNParams; }

int fjb_mlp_forward(const float *params_dev, const float *X_dev, int n, float *Y_dev, void *stream) {
    if (!params_dev || !X_dev || !Y_dev || n < 0) return FJB_E_ARG;
    if (n == 0) return FJB_OK;
    const int grid = std::min((n + 127) / 128, 148 * 8);
    mlp_forward_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(params_dev, X_dev, n, Y_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FJB_OK : rfail("mlp_forward", e);
}

int fjb_mlp_forward_tc(const float *params_dev, const float *X_dev, int n, float *Y_dev, void *stream) {
    if (!params_dev || !X_dev || !Y_dev || n < 0) return FJB_E_ARG;
    if (n == 0) return FJB_OK;
    const int grid = std::min((n + 127) / 128, 148 * 8);
    mlp_forward_tc_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(params_dev, X_dev, n, Y_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FJB_OK : rfail("mlp_forward_tc", e);
}

int fjb_mlp_gradient(const float *params_dev, const float *X_dev, const float *T_dev, int n, float *grad_dev,
                     float *sq_err_dev, float *scratch_dev, void *stream) {
    if (!params_dev || !X_dev || !T_dev || !grad_dev || !sq_err_dev || !scratch_dev || n <= 0) return FJB_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    mlp_fwd_bwd_kernel<<<(n + 127) / 128, 128, 0, st>>>(params_dev, X_dev, T_dev, n, scratch_dev, sq_err_dev);
    mlp_grad_kernel<<<(kNParams + 127) / 128, 128, 0, st>>>(params_dev, X_dev, n, scratch_dev, grad_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FJB_OK : rfail("mlp_gradient", e);
}

int fjb_mlp_adam(float *params_dev, const float *grad_dev, float *m_dev, float *v_dev, float lr, int step,
                 void *stream) {
    if (!params_dev || !grad_dev || !m_dev || !v_dev || step < 1) return FJB_E_ARG;
    mlp_adam_kernel<<<(kNParams + 127) / 128, 128, 0, (cudaStream_t)stream>>>(params_dev, grad_dev, m_dev, v_dev,
                                                                           lr, 0.9f, 0.999f, 1e-8f, step);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FJB_OK : rfail("mlp_adam", e);
}

}  // extern "C"
