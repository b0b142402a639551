"""CPU oracle of Rys quadrature for the two-electron integrals.
TEST INFRASTRUCTURE ONLY: tests/ import it; the product never does.

The reference's third engine (rys/roots.py, rys/recurrence.py) replaces the
HGP VRR by Rys quadrature.  Restated here from the published method, in
plain numpy:

* the rule: the N-point Gauss rule of dmu(x) = (1/2) x^(-1/2) e^(-T x) dx on
  [0, 1] (moments F_m(T)).  With x = t^2 the measure is e^(-T t^2) dt on
  [0, 1]; it is discretised by an M-point Gauss-Legendre rule on [0, b],
  b = min(1, 8 / sqrt(T)) (beyond b the integrand is below e^-64 of its
  start), and the discrete measure's Jacobi matrix comes from the Lanczos
  process with full reorthogonalisation (the discretised Stieltjes
  procedure, Gautschi, Orthogonal Polynomials, 2004, sec. 2.2); nodes are
  its eigenvalues, weights mu_0 times the squared first eigenvector
  components (Golub and Welsch, Math. Comp. 23 (1969) 221).
* the integrals (Rys, Dupuis and King, J. Comput. Chem. 4 (1983) 154): per
  root x and axis, with rho = p q / (p + q),
      C00 = PA - (rho/p) PQ x,  C00' = QC + (rho/q) PQ x,
      B10 = 1/(2p) - rho x/(2 p^2),  B01 = 1/(2q) - rho x/(2 q^2),
      B00 = x / (2 (p + q)),
      I(i+1, k) = C00 I(i, k) + i B10 I(i-1, k) + k B00 I(i, k-1)
      I(i, k+1) = C00' I(i, k) + k B01 I(i, k-1) + i B00 I(i-1, k),
  I(0, 0) = 1; the horizontal transfer I(a, b+1) = I(a+1, b) + AB I(a, b)
  on each side; (ab|cd) = sum over primitive quartets of
  c_a c_b c_c c_d (2 pi^(5/2) / (p q sqrt(p+q))) K_AB K_CD
  sum_n w_n I_x I_y I_z.
"""

from __future__ import annotations

import math

import numpy as np

_GL = {}


def _legendre(m: int):
    if m not in _GL:
        _GL[m] = np.polynomial.legendre.leggauss(m)
    return _GL[m]


def roots_weights(n: int, T: float, m: int = 160):
    """(x, w): the n-point Rys rule at T, nodes ascending."""
    if n < 1:
        raise ValueError("n >= 1")
    T = float(T)
    b = 1.0 if T <= 64.0 else 8.0 / math.sqrt(T)
    s, u = _legendre(m)
    t = 0.5 * b * (s + 1.0)
    y = t * t
    mu = 0.5 * b * u * np.exp(-T * y)
    # Lanczos on diag(y) from the start vector sqrt(mu), fully reorthogonalised
    mu0 = mu.sum()
    q = np.sqrt(mu / mu0)
    Q = [q]
    alpha, beta = [], []
    for k in range(n):
        v = y * Q[-1]
        a = float(Q[-1] @ v)
        alpha.append(a)
        if k == n - 1:
            break
        v = v - a * Q[-1] - (beta[-1] * Q[-2] if beta else 0.0)
        for qq in Q:  # full reorthogonalisation
            v = v - (qq @ v) * qq
        bk = float(np.linalg.norm(v))
        beta.append(bk)
        Q.append(v / bk)
    J = np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1)
    x, V = np.linalg.eigh(J)
    return x, mu0 * V[0] ** 2


def _cart(l):  # noqa: E741
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def _axis(la, lb, lc, ld, pa, qc, pq, ab, cd, p, q, x):
    """I[a, b, c, d] on one axis at root x."""
    rho = p * q / (p + q)
    c00 = pa - rho / p * pq * x
    c00p = qc + rho / q * pq * x
    b10 = 0.5 / p - rho * x / (2.0 * p * p)
    b01 = 0.5 / q - rho * x / (2.0 * q * q)
    b00 = 0.5 * x / (p + q)
    E, F = la + lb, lc + ld
    I = np.zeros((E + 1, F + 1))
    I[0, 0] = 1.0
    for i in range(E):
        I[i + 1, 0] = c00 * I[i, 0] + (i * b10 * I[i - 1, 0] if i else 0.0)
    for k in range(F):
        for i in range(E + 1):
            v = c00p * I[i, k]
            if k:
                v += k * b01 * I[i, k - 1]
            if i:
                v += i * b00 * I[i - 1, k]
            I[i, k + 1] = v
    # horizontal transfer, bra then ket
    X = np.zeros((E + 1, lb + 1, F + 1))
    X[:, 0, :] = I
    for bb in range(lb):
        for a in range(E - bb):
            X[a, bb + 1] = X[a + 1, bb] + ab * X[a, bb]
    Y = np.zeros((la + 1, lb + 1, F + 1, ld + 1))
    Y[:, :, :, 0] = X[:la + 1]
    for dd in range(ld):
        for c in range(F - dd):
            Y[:, :, c, dd + 1] = Y[:, :, c + 1, dd] + cd * Y[:, :, c, dd]
    return Y[:, :, :lc + 1, :]


def eri_block(sa, sb, sc, sd, boys=None) -> np.ndarray:
    """(ab|cd) for shells with l, centre, exponents, coefficients (any
    Shell-like objects), n_cart(a) x n_cart(b) x n_cart(c) x n_cart(d)."""
    A, B, Cc, D = (np.asarray(s.centre, float) for s in (sa, sb, sc, sd))
    la, lb, lc, ld = sa.l, sb.l, sc.l, sd.l
    L = la + lb + lc + ld
    n = L // 2 + 1
    ca_, cb_, cc_, cd_ = _cart(la), _cart(lb), _cart(lc), _cart(ld)
    out = np.zeros((len(ca_), len(cb_), len(cc_), len(cd_)))
    for a1, k1 in zip(sa.exponents, sa.coefficients):
        for a2, k2 in zip(sb.exponents, sb.coefficients):
            p = a1 + a2
            P = (a1 * A + a2 * B) / p
            kab = math.exp(-a1 * a2 / p * float((A - B) @ (A - B)))
            for a3, k3 in zip(sc.exponents, sc.coefficients):
                for a4, k4 in zip(sd.exponents, sd.coefficients):
                    q = a3 + a4
                    Q = (a3 * Cc + a4 * D) / q
                    kcd = math.exp(-a3 * a4 / q * float((Cc - D) @ (Cc - D)))
                    rho = p * q / (p + q)
                    T = rho * float((P - Q) @ (P - Q))
                    pref = k1 * k2 * k3 * k4 * 2.0 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * kab * kcd
                    xs, ws = roots_weights(n, T)
                    for x, w in zip(xs, ws):
                        Ix = _axis(la, lb, lc, ld, P[0] - A[0], Q[0] - Cc[0], P[0] - Q[0], A[0] - B[0],
                                   Cc[0] - D[0], p, q, x)
                        Iy = _axis(la, lb, lc, ld, P[1] - A[1], Q[1] - Cc[1], P[1] - Q[1], A[1] - B[1],
                                   Cc[1] - D[1], p, q, x)
                        Iz = _axis(la, lb, lc, ld, P[2] - A[2], Q[2] - Cc[2], P[2] - Q[2], A[2] - B[2],
                                   Cc[2] - D[2], p, q, x)
                        for i, (ax, ay, az) in enumerate(ca_):
                            for j, (bx, by, bz) in enumerate(cb_):
                                for k, (cx, cy, cz) in enumerate(cc_):
                                    for m, (dx, dy, dz) in enumerate(cd_):
                                        out[i, j, k, m] += pref * w * (Ix[ax, bx, cx, dx] * Iy[ay, by, cy, dy]
                                                                       * Iz[az, bz, cz, dz])
    return out
