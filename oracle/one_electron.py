"""CPU oracle of the one-electron matrices S, T, V and h = T + V.
TEST INFRASTRUCTURE ONLY: tests/ and bench.py's CPU leg import it; the
product (felizjueves_b200) never does.

A restatement, in numpy and plain loops, of the reference's one-electron
path (McMurchie-Davidson):
  * overlap   one_electron/overlap.py:55-66  S_ab = c_a c_b (pi/p)^{3/2}
              E^x_0 E^y_0 E^z_0, E from mmd/hermite.py e_axis (seed
              exp(-mu X_AB^2) per axis);
  * kinetic   one_electron/kinetic.py:61-111  the ket-shift identity
              K_ij = -2 b^2 S_{i,j+2} + b (2j+1) S_{i,j} - j(j-1)/2 S_{i,j-2},
              T = K_x S_y S_z + S_x K_y S_z + S_x S_y K_z;
  * potential one_electron/potential.py:1-60, 79-110  V_ab = -sum_C Z_C
              (2 pi / p) sum_tuv E^x_t E^y_u E^z_v R_tuv(p, P - C), R the
              Hermite Coulomb integrals from (-2p)^n F_n(p |PC|^2);
  * assembly  one_electron/one_electron.py:57-110  every unordered shell
              pair once, the diagonal blocks' upper triangle mirrored, so
              each matrix is exactly symmetric.
Boys values come from the pinned C oracle (`oracle.boys`).  Shell
coefficients multiply unnormalised primitives (ao/shell.py).
"""

from __future__ import annotations

import math

import numpy as np

from . import oracle


def _cartesians(l):  # noqa: E741
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def e_table(la, lb, p, pa, pb, seed):
    """E[i][j][t], i <= la, j <= lb, t <= i + j (mmd/hermite.py e_axis)."""
    E = np.zeros((la + 1, lb + 1, la + lb + 2))
    E[0, 0, 0] = seed
    h = 0.5 / p
    for j in range(lb):
        for t in range(j + 2):
            v = pb * E[0, j, t] + (t + 1) * E[0, j, t + 1]
            if t > 0:
                v += h * E[0, j, t - 1]
            E[0, j + 1, t] = v
    for i in range(la):
        for j in range(lb + 1):
            for t in range(i + j + 2):
                v = pa * E[i, j, t] + (t + 1) * E[i, j, t + 1]
                if t > 0:
                    v += h * E[i, j, t - 1]
                E[i + 1, j, t] = v
    return E


def r_table(L, p, pc, F):
    """R[t][u][v] = R^0_tuv for t + u + v <= L, from F[n] = F_n(p |PC|^2)."""
    Rn1 = None
    for n in range(L, -1, -1):
        Rn = np.zeros((L + 1, L + 1, L + 1))
        for s in range(L - n + 1):
            for t in range(s, -1, -1):
                for u in range(s - t, -1, -1):
                    v = s - t - u
                    if s == 0:
                        Rn[0, 0, 0] = (-2.0 * p) ** n * F[n]
                    elif t > 0:
                        Rn[t, u, v] = pc[0] * Rn1[t - 1, u, v] + ((t - 1) * Rn1[t - 2, u, v] if t > 1 else 0.0)
                    elif u > 0:
                        Rn[t, u, v] = pc[1] * Rn1[t, u - 1, v] + ((u - 1) * Rn1[t, u - 2, v] if u > 1 else 0.0)
                    else:
                        Rn[t, u, v] = pc[2] * Rn1[t, u, v - 1] + ((v - 1) * Rn1[t, u, v - 2] if v > 1 else 0.0)
        Rn1 = Rn
    return Rn1


def blocks(sa, sb, nuclei):
    """(S, T, V) blocks of one shell pair: n_cart(sa) x n_cart(sb) each."""
    A, B = np.asarray(sa.centre), np.asarray(sb.centre)
    la, lb = sa.l, sb.l
    ca_, cb_ = _cartesians(la), _cartesians(lb)
    S = np.zeros((len(ca_), len(cb_)))
    T = np.zeros_like(S)
    V = np.zeros_like(S)
    for a, ca in zip(sa.exponents, sa.coefficients):
        for b, cb in zip(sb.exponents, sb.coefficients):
            p = a + b
            mu = a * b / p
            P = (a * A + b * B) / p
            Es = []  # per axis, ket widened to lb + 2 for the kinetic shift
            for d in range(3):
                seed = math.exp(-mu * (A[d] - B[d]) ** 2)
                Es.append(e_table(la, lb + 2, p, P[d] - A[d], P[d] - B[d], seed))
            dress = ca * cb * (math.pi / p) ** 1.5
            for r, ax in enumerate(ca_):
                for c, bx in enumerate(cb_):
                    s = [Es[d][ax[d], bx[d], 0] for d in range(3)]
                    k = []
                    for d in range(3):
                        j = bx[d]
                        row = Es[d][ax[d], :, 0]
                        kk = -2.0 * b * b * row[j + 2] + b * (2 * j + 1) * row[j]
                        if j >= 2:
                            kk -= 0.5 * j * (j - 1) * row[j - 2]
                        k.append(kk)
                    S[r, c] += dress * s[0] * s[1] * s[2]
                    T[r, c] += dress * (k[0] * s[1] * s[2] + s[0] * k[1] * s[2] + s[0] * s[1] * k[2])
            L = la + lb
            pref = ca * cb * 2.0 * math.pi / p
            for Z, C in nuclei:
                pc = P - np.asarray(C, float)
                x = p * float(pc @ pc)
                F = [oracle.boys(n, x) for n in range(L + 1)]
                R = r_table(L, p, pc, F)
                for r, ax in enumerate(ca_):
                    for c, bx in enumerate(cb_):
                        acc = 0.0
                        for t in range(ax[0] + bx[0] + 1):
                            for u in range(ax[1] + bx[1] + 1):
                                for v in range(ax[2] + bx[2] + 1):
                                    acc += (Es[0][ax[0], bx[0], t] * Es[1][ax[1], bx[1], u]
                                            * Es[2][ax[2], bx[2], v] * R[t, u, v])
                        V[r, c] += -Z * pref * acc
    return S, T, V


def matrices(basis, nuclei):
    """(S, T, V), each n_ao x n_ao and exactly symmetric."""
    n = basis.n_ao
    out = [np.zeros((n, n)) for _ in range(3)]
    sh, off = basis.shells, basis.offsets
    for i in range(len(sh)):
        for j in range(i, len(sh)):
            bl = blocks(sh[i], sh[j], nuclei)
            oa, ob = off[i], off[j]
            for M, b in zip(out, bl):
                for r in range(b.shape[0]):
                    for c in range(b.shape[1]):
                        if i == j and c < r:
                            continue
                        M[oa + r, ob + c] = b[r, c]
                        M[ob + c, oa + r] = b[r, c]
    return tuple(out)
