// rys_table.cpp -- the Chebyshev table behind rys_rule (rys_rule.h).
//
// At each interval's Chebyshev points the n-point rule is computed in long
// double (64-bit mantissa) by the discretised Stieltjes procedure (Gautschi,
// Orthogonal Polynomials, 2004, sec. 2.2): with x = t^2 the measure is
// e^(-T t^2) dt on [0, 1] (or [0, 10/sqrt(T)] where that is shorter: the rest
// is below e^-100), discretised by a kRysQuad-point Gauss-Legendre rule; the Lanczos process on it (fully reorthogonalised) gives the Jacobi
// matrix, whose eigenvalues are the nodes and whose eigenvectors' first
// components squared, times the measure's mass, the weights (Golub and
// Welsch, Math. Comp. 23 (1969) 221).  The small symmetric eigenproblems are
// solved by cyclic Jacobi rotations.  The rule's values at the points are
// fitted by the discrete Chebyshev transform, rounded once to double.  The
// asymptotic constants are the generalised Gauss-Laguerre rule for the
// weight y^(-1/2) e^(-y), from its three-term recurrence
// (a_k = 2k + 1/2, b_k = k (k - 1/2), mass Gamma(1/2)).
#include <algorithm>
#include <cmath>
#include <vector>

#include "rys_rule.h"

namespace fjb {

namespace {

using LD = long double;
constexpr LD kPiL = 3.141592653589793238462643383279502884L;
constexpr int kRysQuad = 200;

void gauss_legendre(int m, std::vector<LD> *t, std::vector<LD> *u) {
    t->assign(m, 0.0L);
    u->assign(m, 0.0L);
    for (int i = 0; i < m; ++i) {
        LD z = cosl(kPiL * ((LD)i + 0.75L) / ((LD)m + 0.5L)), dp = 1.0L;
        for (int it = 0; it < 100; ++it) {
            LD p0 = 1.0L, p1 = z;
            for (int k = 2; k <= m; ++k) {
                const LD p2 = ((LD)(2 * k - 1) * z * p1 - (LD)(k - 1) * p0) / (LD)k;
                p0 = p1;
                p1 = p2;
            }
            dp = (LD)m * (z * p1 - p0) / (z * z - 1.0L);
            const LD dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-19L) break;
        }
        LD p0 = 1.0L, p1 = z;
        for (int k = 2; k <= m; ++k) {
            const LD p2 = ((LD)(2 * k - 1) * z * p1 - (LD)(k - 1) * p0) / (LD)k;
            p0 = p1;
            p1 = p2;
        }
        dp = (LD)m * (z * p1 - p0) / (z * z - 1.0L);
        (*t)[i] = z;
        (*u)[i] = 2.0L / ((1.0L - z * z) * dp * dp);
    }
}

// Eigenvalues (ascending) of the symmetric n x n matrix A and the first
// component of each unit eigenvector, by cyclic Jacobi rotations.
void jacobi_eig(int n, std::vector<LD> A, LD *ev, LD *first) {
    std::vector<LD> V((size_t)n * n, 0.0L);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0L;
    auto a = [&](int i, int j) -> LD & { return A[(size_t)i * n + j]; };
    auto v = [&](int i, int j) -> LD & { return V[(size_t)i * n + j]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        LD off = 0.0L, diag = 0.0L;
        for (int p = 0; p < n; ++p) {
            diag += a(p, p) * a(p, p);
            for (int q = p + 1; q < n; ++q) off += a(p, q) * a(p, q);
        }
        if (off <= 1e-40L * diag || off == 0.0L) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                if (a(p, q) == 0.0L) continue;
                const LD th = (a(q, q) - a(p, p)) / (2.0L * a(p, q));
                const LD t = (th >= 0.0L ? 1.0L : -1.0L) / (fabsl(th) + sqrtl(th * th + 1.0L));
                const LD c = 1.0L / sqrtl(t * t + 1.0L), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const LD kp = a(k, p), kq = a(k, q);
                    a(k, p) = c * kp - s * kq;
                    a(k, q) = s * kp + c * kq;
                }
                for (int k = 0; k < n; ++k) {
                    const LD pk = a(p, k), qk = a(q, k);
                    a(p, k) = c * pk - s * qk;
                    a(q, k) = s * pk + c * qk;
                }
                for (int k = 0; k < n; ++k) {
                    const LD kp = v(k, p), kq = v(k, q);
                    v(k, p) = c * kp - s * kq;
                    v(k, q) = s * kp + c * kq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int i, int j) { return a(i, i) < a(j, j); });
    for (int i = 0; i < n; ++i) {
        ev[i] = a(idx[i], idx[i]);
        first[i] = v(0, idx[i]);
    }
}

// The n-point Gauss rule of the (discretised) measure at T.
void rule_at(int n, LD T, const std::vector<LD> &gt, const std::vector<LD> &gu, LD *x, LD *w) {
    const int m = (int)gt.size();
    // [0, b]: beyond t = 10/sqrt(T) the density is below e^-100 of its start
    const LD b = T > 100.0L ? 10.0L / sqrtl(T) : 1.0L;
    std::vector<LD> y(m), mu(m);
    LD mu0 = 0.0L;
    for (int j = 0; j < m; ++j) {
        const LD t = 0.5L * b * (gt[j] + 1.0L);
        y[j] = t * t;
        mu[j] = 0.5L * b * gu[j] * expl(-T * y[j]);
        mu0 += mu[j];
    }
    std::vector<std::vector<LD>> Q;
    std::vector<LD> q(m), alpha, beta;
    for (int j = 0; j < m; ++j) q[j] = sqrtl(mu[j] / mu0);
    Q.push_back(q);
    for (int k = 0; k < n; ++k) {
        const std::vector<LD> &qk = Q.back();
        std::vector<LD> vv(m);
        LD ak = 0.0L;
        for (int j = 0; j < m; ++j) {
            vv[j] = y[j] * qk[j];
            ak += qk[j] * vv[j];
        }
        alpha.push_back(ak);
        if (k == n - 1) break;
        for (int pass = 0; pass < 2; ++pass)  // full reorthogonalisation, twice (covers alpha and beta)
            for (const auto &qq : Q) {
                LD d = 0.0L;
                for (int j = 0; j < m; ++j) d += qq[j] * vv[j];
                for (int j = 0; j < m; ++j) vv[j] -= d * qq[j];
            }
        LD bk = 0.0L;
        for (int j = 0; j < m; ++j) bk += vv[j] * vv[j];
        bk = sqrtl(bk);
        beta.push_back(bk);
        for (int j = 0; j < m; ++j) vv[j] /= bk;
        Q.push_back(vv);
    }
    std::vector<LD> J((size_t)n * n, 0.0L);
    for (int i = 0; i < n; ++i) J[(size_t)i * n + i] = alpha[i];
    for (int i = 0; i + 1 < n; ++i) J[(size_t)i * n + i + 1] = J[(size_t)(i + 1) * n + i] = beta[i];
    std::vector<LD> f(n);
    jacobi_eig(n, J, x, f.data());
    for (int i = 0; i < n; ++i) w[i] = mu0 * f[i] * f[i];
}

}  // namespace

std::vector<double> rys_table() {
    std::vector<double> tab(kRysTableSize, 0.0);
    std::vector<LD> gt, gu;
    gauss_legendre(kRysQuad, &gt, &gu);
    const int P = kRysDeg + 1;
    std::vector<LD> xs((size_t)P * kRysMaxN), ws((size_t)P * kRysMaxN);
    for (int n = 1; n <= kRysMaxN; ++n)
        for (int i = 0; i < kRysNI; ++i) {
            const LD a = (LD)i * (LD)kRysWidth;
            for (int j = 0; j < P; ++j) {
                const LD uj = cosl(kPiL * ((LD)j + 0.5L) / (LD)P);
                rule_at(n, a + 0.5L * (uj + 1.0L) * (LD)kRysWidth, gt, gu, &xs[(size_t)j * kRysMaxN],
                        &ws[(size_t)j * kRysMaxN]);
            }
            double *blk = tab.data() + ((size_t)(n - 1) * kRysNI + i) * kRysBlock;
            for (int r = 0; r < n; ++r)
                for (int k = 0; k < P; ++k) {
                    LD cx = 0.0L, cw = 0.0L;
                    for (int j = 0; j < P; ++j) {
                        const LD ck = cosl(kPiL * (LD)k * ((LD)j + 0.5L) / (LD)P);
                        cx += xs[(size_t)j * kRysMaxN + r] * ck;
                        cw += ws[(size_t)j * kRysMaxN + r] * ck;
                    }
                    const LD s = (k == 0 ? 1.0L : 2.0L) / (LD)P;
                    blk[(2 * r) * P + k] = (double)(cx * s);
                    blk[(2 * r + 1) * P + k] = (double)(cw * s);
                }
        }
    // the asymptotic rule: generalised Gauss-Laguerre, alpha = -1/2
    for (int n = 1; n <= kRysMaxN; ++n) {
        std::vector<LD> J((size_t)n * n, 0.0L);
        for (int k = 0; k < n; ++k) J[(size_t)k * n + k] = 2.0L * (LD)k + 0.5L;
        for (int k = 1; k < n; ++k) J[(size_t)(k - 1) * n + k] = J[(size_t)k * n + k - 1] = sqrtl((LD)k * ((LD)k - 0.5L));
        std::vector<LD> s(n), f(n);
        jacobi_eig(n, J, s.data(), f.data());
        double *a = tab.data() + kRysAsym + (size_t)(n - 1) * kRysMaxN * 2;
        for (int r = 0; r < n; ++r) {
            a[2 * r] = (double)s[r];
            a[2 * r + 1] = (double)(sqrtl(kPiL) * f[r] * f[r]);
        }
    }
    return tab;
}

}  // namespace fjb
