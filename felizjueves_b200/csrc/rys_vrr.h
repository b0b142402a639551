// rys_vrr.h -- the Rys replacement of the HGP VRR (host/device functions).
//
// One primitive quartet's boundary [e0|f0]^(0) (e on the bra centre A with
// la <= |e| <= la + lb, f on the ket centre C with lc <= |f| <= lc + ld: the
// values the HGP HRR reads) by Rys quadrature instead of the vertical
// recurrence, as the reference's third engine does (rys/recurrence.py,
// eri/fock/kernel_frys.py):
//
//   [e0|f0] = seed sum_n w_n I_x(e_x, f_x) I_y(e_y, f_y) I_z(e_z, f_z),
//   seed = U_P U_Q (2/sqrt(pi)) sqrt(rho),  (w_n, x_n) the n-point rule at T,
//
// with the 2D integrals of each axis from the Rys-Dupuis-King recurrences
// (J. Comput. Chem. 4 (1983) 154) at root x:
//
//   C00 = PA - (rho/p) PQ x,  C00' = QC + (rho/q) PQ x,
//   B10 = (1 - (rho/p) x) / (2p),  B01 = (1 - (rho/q) x) / (2q),  B00 = x / (2(p+q)),
//   I(i+1, 0) = C00 I(i, 0) + i B10 I(i-1, 0),
//   I(i, k+1) = C00' I(i, k) + k B01 I(i, k-1) + i B00 I(i-1, k),  I(0, 0) = 1.
#pragma once
#include "rys_rule.h"

namespace fjb {

constexpr int kRysMaxE = 7;  // la + lb + 1 and lc + ld + 1 for l <= 3

// I[i][k], i <= E, k <= F, of one axis at one root.
FJB_HD inline void rys_axis(int E, int F, double c00, double c00p, double b10, double b01, double b00,
                            double I[kRysMaxE][kRysMaxE]) {
    I[0][0] = 1.0;
    for (int i = 0; i < E; ++i) I[i + 1][0] = c00 * I[i][0] + (i ? (double)i * b10 * I[i - 1][0] : 0.0);
    for (int k = 0; k < F; ++k)
        for (int i = 0; i <= E; ++i) {
            double v = c00p * I[i][k];
            if (k) v += (double)k * b01 * I[i][k - 1];
            if (i) v += (double)i * b00 * I[i - 1][k];
            I[i][k + 1] = v;
        }
}

// The n-point rule's roots and the three axes' tables of one primitive
// quartet: P, Q its centres, A, C the bra and ket shell centres.
// I[r][d] is root r's table on axis d.
FJB_HD inline void rys_tables(int E, int F, double p, double q, const double *P, const double *Q, const double *A,
                              const double *C, const double *tab, double *w, double I[][3][kRysMaxE][kRysMaxE]) {
    const int n = (E + F) / 2 + 1;
    const double rho = p * q / (p + q);
    const double PQ[3] = {P[0] - Q[0], P[1] - Q[1], P[2] - Q[2]};
    const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    double x[kRysMaxN];
    rys_rule(n, T, tab, x, w);
    for (int r = 0; r < n; ++r) {
        const double b10 = (1.0 - rho / p * x[r]) / (2.0 * p), b01 = (1.0 - rho / q * x[r]) / (2.0 * q);
        const double b00 = x[r] / (2.0 * (p + q));
        for (int d = 0; d < 3; ++d)
            rys_axis(E, F, (P[d] - A[d]) - rho / p * PQ[d] * x[r], (Q[d] - C[d]) + rho / q * PQ[d] * x[r], b10,
                     b01, b00, I[r][d]);
    }
}

}  // namespace fjb
