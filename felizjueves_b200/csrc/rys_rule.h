// rys_rule.h -- the tabulated Rys rule (host table, host/device evaluation).
//
// The n-point Gauss rule of dmu(x) = (1/2) x^(-1/2) e^(-T x) dx on [0, 1]
// (its moments are the Boys values F_m(T), m <= 2n - 1), n = 1..kRysMaxN
// (kRysMaxN = 7 reaches (ff|ff), L = 12): the quadrature a Rys VRR runs per
// primitive quartet (the reference's rys/roots.py computes the same rule by
// Stieltjes + bisection per call; here it is a table lookup).
//
// Below kRysTSwitch each node and weight is a Chebyshev series of degree
// kRysDeg on intervals of width kRysWidth (rys_table.cpp builds it);
// above, the rule is the generalised Gauss-Laguerre one (alpha = -1/2)
// scaled, x = s / T, w = v / (2 sqrt(T)), whose dropped tail is below
// e^-T of the rule.
#pragma once
#include <cmath>
#include <vector>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define FJB_HD __host__ __device__
#else
#define FJB_HD
#endif

namespace fjb {

constexpr int kRysMaxN = 7;
// The asymptote's relative error is about e^-T T^(2n - 3/2): below 1e-29 at
// T = 128 for n = 7 (at T = 64 it would be 6e-6).
constexpr double kRysTSwitch = 128.0;
constexpr double kRysWidth = 1.0;
constexpr int kRysNI = 128;  // kRysTSwitch / kRysWidth intervals
constexpr int kRysDeg = 15;  // Chebyshev degree per interval
constexpr int kRysBlock = kRysMaxN * 2 * (kRysDeg + 1);  // one (n, interval): roots x (x, w) x coefficients
constexpr int kRysAsym = kRysMaxN * kRysNI * kRysBlock;  // offset of the (s, v) constants
constexpr int kRysTableSize = kRysAsym + kRysMaxN * kRysMaxN * 2;

// The table: [n-1][interval][root][x | w][Chebyshev coefficient], then
// [n-1][root][s | v].  Built once, on the host.
std::vector<double> rys_table();

FJB_HD inline double rys_clenshaw(const double *c, double u) {
    double b1 = 0.0, b2 = 0.0;
    for (int k = kRysDeg; k >= 1; --k) {
        const double b0 = 2.0 * u * b1 - b2 + c[k];
        b2 = b1;
        b1 = b0;
    }
    return u * b1 - b2 + c[0];
}

// Nodes x[0..n-1] (ascending) and weights w[0..n-1] at T >= 0.
FJB_HD inline void rys_rule(int n, double T, const double *tab, double *x, double *w) {
    if (T < kRysTSwitch) {
        int i = (int)(T * (1.0 / kRysWidth));
        if (i > kRysNI - 1) i = kRysNI - 1;
        const double u = 2.0 * (T - (double)i * kRysWidth) * (1.0 / kRysWidth) - 1.0;
        const double *blk = tab + ((size_t)(n - 1) * kRysNI + i) * kRysBlock;
        for (int r = 0; r < n; ++r) {
            x[r] = rys_clenshaw(blk + (2 * r) * (kRysDeg + 1), u);
            w[r] = rys_clenshaw(blk + (2 * r + 1) * (kRysDeg + 1), u);
        }
    } else {
        const double it = 1.0 / T, hs = 0.5 / sqrt(T);
        const double *a = tab + kRysAsym + (size_t)(n - 1) * kRysMaxN * 2;
        for (int r = 0; r < n; ++r) {
            x[r] = a[2 * r] * it;
            w[r] = a[2 * r + 1] * hs;
        }
    }
}

}  // namespace fjb
