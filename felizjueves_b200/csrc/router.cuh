// router.cuh -- the learned precision router: quartet features and the MLP.
//
// Features of a quartet (12, FP32): log zeta and log eta of the pairs'
// leading (largest-bound) primitive pairs, |AB|, |CD|, the distance between
// those primitives' centres P and Q, la, lb, lc, ld, log10 G_ab, log10 G_cd,
// log10 of the six-block weighted density maximum (the screen's dmax).
// The network: 12 -> 64 -> 64 -> 1, tanh hidden layers, standardised inputs,
// and a fixed skip connection: the output is log10 G_ab + log10 G_cd +
// log10 dmax (the Schwarz x density bound, features 9-11) plus the network's
// value, so the network itself learns the gap between the quartet's largest
// deposit (max |ERI| x dmax) and that bound.  Parameters, FP32, packed as
//   mu[12] sd[12] W1[64][12] b1[64] W2[64][64] b2[64] w3[64] b3
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fjb_internal.h"

namespace fjb {

constexpr int kFeat = 12, kHid = 64;
constexpr int kOffMu = 0, kOffSd = kOffMu + kFeat, kOffW1 = kOffSd + kFeat, kOffB1 = kOffW1 + kHid * kFeat,
              kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid,
              kOffB3 = kOffW3 + kHid, kNParams = kOffB3 + 1;

__device__ __forceinline__ float safe_log10(double x) { return (float)log10(fmax(x, 1e-300)); }

__device__ __forceinline__ void quartet_features(const PairRec &bra, const PairRec &ket, const PrimRec *prims,
                                                 int la, int lb, int lc, int ld, double dmax, float *f) {
    const PrimRec P = prims[bra.prim0], Q = prims[ket.prim0];
    f[0] = (float)log(P.zeta);
    f[1] = (float)log(Q.zeta);
    f[2] = (float)sqrt(bra.AB[0] * bra.AB[0] + bra.AB[1] * bra.AB[1] + bra.AB[2] * bra.AB[2]);
    f[3] = (float)sqrt(ket.AB[0] * ket.AB[0] + ket.AB[1] * ket.AB[1] + ket.AB[2] * ket.AB[2]);
    const double dx = P.P[0] - Q.P[0], dy = P.P[1] - Q.P[1], dz = P.P[2] - Q.P[2];
    f[4] = (float)sqrt(dx * dx + dy * dy + dz * dz);
    f[5] = (float)la;
    f[6] = (float)lb;
    f[7] = (float)lc;
    f[8] = (float)ld;
    f[9] = safe_log10(bra.G);
    f[10] = safe_log10(ket.G);
    f[11] = safe_log10(dmax);
}

// The six-block weighted density maximum (the screen's dmax).
__device__ __forceinline__ double six_block_dmax(const double *__restrict__ Dsh, int n_sh, int a, int b, int c,
                                                 int d) {
    double dmax = 2.0 * __ldg(Dsh + (size_t)a * n_sh + b);
    double t = 2.0 * __ldg(Dsh + (size_t)c * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + d);
    if (dmax < t) dmax = t;
    return dmax;
}

// Forward pass of one sample; p points at the packed parameters (shared or
// global).  h1, h2 receive the hidden activations when non-null.
__device__ __forceinline__ float mlp_forward(const float *__restrict__ p, const float *x, float *h1, float *h2) {
    float xn[kFeat];
#pragma unroll
    for (int i = 0; i < kFeat; ++i) xn[i] = (x[i] - p[kOffMu + i]) / p[kOffSd + i];
    float a1[kHid];
#pragma unroll 8
    for (int j = 0; j < kHid; ++j) {
        float s = p[kOffB1 + j];
#pragma unroll
        for (int i = 0; i < kFeat; ++i) s += p[kOffW1 + j * kFeat + i] * xn[i];
        a1[j] = tanhf(s);
    }
    float y = p[kOffB3] + (x[9] + x[10] + x[11]);
#pragma unroll 4
    for (int k = 0; k < kHid; ++k) {
        float s = p[kOffB2 + k];
#pragma unroll 8
        for (int j = 0; j < kHid; ++j) s += p[kOffW2 + k * kHid + j] * a1[j];
        const float hk = tanhf(s);
        if (h2) h2[k] = hk;
        y += p[kOffW3 + k] * hk;
    }
    if (h1)
        for (int j = 0; j < kHid; ++j) h1[j] = a1[j];
    return y;
}

// The forward pass of a warp's 32 samples on the tensor cores (the router's
// inference: its margin is calibrated through this same arithmetic,
// fjb_mlp_forward_tc).  Both hidden layers are mma.sync m16n8k16 products
// with FP16 operands and FP32 accumulation, rows = the warp's samples (two
// 16-row tiles), the hidden units 8-column tiles; a layer's accumulator
// tiles are the next layer's operand fragments as they stand (columns
// 16 kb .. 16 kb + 15 of layer 1 are n-tiles 2 kb and 2 kb + 1), so
// nothing goes back through memory; tanh by the hardware's approximation.
// The half-precision weights, staged once per CTA: w1h[n][k] = W1[n][k]
// (k padded to 16 with zeros), w2h[n][j] = W2[n][j]; xs is this warp's
// 32-row half staging of its standardised inputs.  Rows are padded (24, 72
// and 24 halves) so that a fragment's eight row groups fall in distinct
// banks.  Every lane of the warp calls it, converged, with its own sample x
// (any finite values where the lane has none) and receives its prediction.
constexpr int kW1Row = 24, kW2Row = 72, kXRow = 24;  // halves
constexpr int kTcSmemHalves = kHid * kW1Row + kHid * kW2Row;  // + 32 kXRow a warp
__device__ __forceinline__ unsigned pack_half2(float lo, float hi) {
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&h);
}

__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void mma_16816(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Stage the hidden layers' weights in FP16 (every thread of the CTA calls it;
// a barrier must follow before use).
__device__ __forceinline__ void stage_mlp_half(const float *__restrict__ p, __half *w1h, __half *w2h) {
    for (int i = threadIdx.x; i < kHid * kW1Row; i += blockDim.x) {
        const int n = i / kW1Row, k = i % kW1Row;
        w1h[i] = __float2half_rn(k < kFeat ? p[kOffW1 + n * kFeat + k] : 0.f);
    }
    for (int i = threadIdx.x; i < kHid * kW2Row; i += blockDim.x) {
        const int n = i / kW2Row, j = i % kW2Row;
        w2h[i] = __float2half_rn(j < kHid ? p[kOffW2 + n * kHid + j] : 0.f);
    }
}

__device__ __forceinline__ float mlp_forward_tc(const float *__restrict__ p, const __half *__restrict__ w1h,
                                                const __half *__restrict__ w2h, __half *xs, const float *x) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    unsigned *xrow = reinterpret_cast<unsigned *>(xs) + lane * (kXRow / 2);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int k0 = 2 * i, k1 = 2 * i + 1;
        xrow[i] = pack_half2(k0 < kFeat ? (x[k0] - p[kOffMu + k0]) / p[kOffSd + k0] : 0.f,
                             k1 < kFeat ? (x[k1] - p[kOffMu + k1]) / p[kOffSd + k1] : 0.f);
    }
    __syncwarp();
    constexpr int XW = kXRow / 2, W1W = kW1Row / 2, W2W = kW2Row / 2;  // row strides in 32-bit words
    const unsigned *xw = reinterpret_cast<const unsigned *>(xs);
    const unsigned *w1w = reinterpret_cast<const unsigned *>(w1h);
    const unsigned *w2w = reinterpret_cast<const unsigned *>(w2h);
    unsigned h1[2][8][2];  // layer 1's tanh, packed: [m-tile][n-tile][row g, row g + 8]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = 16 * mt + g;
        const unsigned a[4] = {xw[r0 * XW + t], xw[(r0 + 8) * XW + t], xw[r0 * XW + 4 + t], xw[(r0 + 8) * XW + 4 + t]};
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int n = 8 * nt + g;
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma_16816(c, a, w1w[n * W1W + t], w1w[n * W1W + 4 + t]);
            const float b0 = p[kOffB1 + 8 * nt + 2 * t], b1 = p[kOffB1 + 8 * nt + 2 * t + 1];
            h1[mt][nt][0] = pack_half2(tanh_approx(c[0] + b0), tanh_approx(c[1] + b1));
            h1[mt][nt][1] = pack_half2(tanh_approx(c[2] + b0), tanh_approx(c[3] + b1));
        }
    }
    float part[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [m-tile][row g, row g + 8]
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int n = 8 * nt + g, col = 8 * nt + 2 * t;
        const float bb0 = p[kOffB2 + col], bb1 = p[kOffB2 + col + 1];
        const float w30 = p[kOffW3 + col], w31 = p[kOffW3 + col + 1];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kb = 0; kb < 4; ++kb) {
                const unsigned a[4] = {h1[mt][2 * kb][0], h1[mt][2 * kb][1], h1[mt][2 * kb + 1][0],
                                       h1[mt][2 * kb + 1][1]};
                mma_16816(c, a, w2w[n * W2W + 8 * kb + t], w2w[n * W2W + 8 * kb + 4 + t]);
            }
            part[mt][0] += w30 * tanh_approx(c[0] + bb0) + w31 * tanh_approx(c[1] + bb1);
            part[mt][1] += w30 * tanh_approx(c[2] + bb0) + w31 * tanh_approx(c[3] + bb1);
        }
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            part[mt][h] += __shfl_xor_sync(0xffffffffu, part[mt][h], 1);
            part[mt][h] += __shfl_xor_sync(0xffffffffu, part[mt][h], 2);
        }
    // row r = 16 mt + 8 h + g' is summed on lane 4 g'
    const int src = 4 * (lane & 7), mt = lane >> 4, h = (lane >> 3) & 1;
    const float v00 = __shfl_sync(0xffffffffu, part[0][0], src), v01 = __shfl_sync(0xffffffffu, part[0][1], src);
    const float v10 = __shfl_sync(0xffffffffu, part[1][0], src), v11 = __shfl_sync(0xffffffffu, part[1][1], src);
    const float y = mt ? (h ? v11 : v10) : (h ? v01 : v00);
    __syncwarp();  // xs is read by every lane before a next call rewrites it
    return y + p[kOffB3] + (x[9] + x[10] + x[11]);
}

}  // namespace fjb
