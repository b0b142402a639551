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

}  // namespace fjb
