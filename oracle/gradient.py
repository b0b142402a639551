"""CPU oracle of the J and K terms of the nuclear gradient of G.
TEST INFRASTRUCTURE ONLY: tests/ import it; the product never does.

The derivative integrals (d_x a b|c d), d_x acting on the electron
coordinate of the first function, by the Cartesian shift identity

    d/dx [x_A^i e^(-alpha r_A^2)] = i x_A^(i-1) e^(...) - 2 alpha x_A^(i+1) e^(...)

so a shell's derivative is a shell of l + 1 with coefficients c (-2 alpha)
plus i times a shell of l - 1 with coefficients c; each is an ordinary ERI
block of the pinned C oracle (`oracle.eri_block`, the reference's
eri/eri.py:86-145 restated).  Contracted as PySCF's grad.rhf.get_jk does
over libcint's int2e_ip1 (the reference's gradient fixtures record its
output; the reference's own path is gradient/kernel_gf.py):

    vj1[x, i, j] = -sum_kl (d_x i j|k l) D[l, k]
    vk1[x, i, l] = -sum_jk (d_x i j|k l) D[j, k]

and per atom A, over the AOs i on A,

    grad_J[A, x] = 2 sum_(i on A) sum_j vj1[x, i, j] D[i, j]
    grad_K[A, x] = 2 sum_(i on A) sum_j (-1/2) vk1[x, i, j] D[i, j].
"""

from __future__ import annotations

import numpy as np

from . import oracle


def _carts(l):  # noqa: E741
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def derivative_eri(basis) -> np.ndarray:
    """dE[x, i, j, k, l] = (d_x i j|k l) over every AO, n^4 x 3."""
    f = basis.flat()
    ns = len(f["l"])
    l0 = [int(x) for x in f["l"]]
    # augmented basis: the shells, then each shell at l + 1 with c (-2 alpha),
    # then each shell with l >= 1 at l - 1 with c
    L, cen, p0, npr, ex, co = [], [], [], [], [], []

    def add(l, c, e, k):  # noqa: E741
        L.append(l)
        cen.append(c)
        p0.append(len(ex))
        npr.append(len(e))
        ex.extend(e)
        co.extend(k)

    for s in range(ns):
        a, n = int(f["prim0"][s]), int(f["nprim"][s])
        add(l0[s], f["centre"][s], f["exps"][a:a + n], f["coefs"][a:a + n])
    for s in range(ns):
        a, n = int(f["prim0"][s]), int(f["nprim"][s])
        e = f["exps"][a:a + n]
        add(l0[s] + 1, f["centre"][s], e, -2.0 * e * f["coefs"][a:a + n])
    minus = {}
    for s in range(ns):
        if l0[s] >= 1:
            a, n = int(f["prim0"][s]), int(f["nprim"][s])
            minus[s] = len(L)
            add(l0[s] - 1, f["centre"][s], f["exps"][a:a + n], f["coefs"][a:a + n])
    ob = oracle.OracleBasis(L, np.asarray(cen).reshape(-1, 3), p0, npr, ex, co)
    off = [int(x) for x in f["ao_off"]]
    nao = basis.n_ao
    nc = [len(_carts(l)) for l in l0]
    out = np.zeros((3, nao, nao, nao, nao))
    for A in range(ns):
        la = l0[A]
        up = {c: k for k, c in enumerate(_carts(la + 1))}
        dn = {c: k for k, c in enumerate(_carts(la - 1))} if la >= 1 else {}
        for B in range(ns):
            for Cs in range(ns):
                for Ds in range(ns):
                    shp = (nc[B], nc[Cs], nc[Ds])
                    bp = oracle.eri_block(ob, ns + A, B, Cs, Ds).reshape((len(up),) + shp)
                    bm = (oracle.eri_block(ob, minus[A], B, Cs, Ds).reshape((len(dn),) + shp)
                          if la >= 1 else None)
                    for r, comp in enumerate(_carts(la)):
                        for x in range(3):
                            cp = list(comp)
                            cp[x] += 1
                            v = bp[up[tuple(cp)]].copy()
                            if comp[x] > 0:
                                cm = list(comp)
                                cm[x] -= 1
                                v += comp[x] * bm[dn[tuple(cm)]]
                            out[x, off[A] + r, off[B]:off[B] + nc[B], off[Cs]:off[Cs] + nc[Cs],
                                off[Ds]:off[Ds] + nc[Ds]] = v
    return out


def jk_derivatives(basis, D):
    """(vj1, vk1), each 3 x n x n, in grad.rhf.get_jk's convention."""
    dE = derivative_eri(basis)
    vj1 = -np.einsum("xijkl,lk->xij", dE, D)
    vk1 = -np.einsum("xijkl,jk->xil", dE, D)
    return vj1, vk1


def gradient_jk(vj1, vk1, D, ao_atom, n_atoms):
    """(grad_J, grad_K), each n_atoms x 3."""
    gj = np.zeros((n_atoms, 3))
    gk = np.zeros((n_atoms, 3))
    for i, a in enumerate(ao_atom):
        gj[a] += 2.0 * np.einsum("xj,j->x", vj1[:, i, :], D[i, :])
        gk[a] += 2.0 * np.einsum("xj,j->x", -0.5 * vk1[:, i, :], D[i, :])
    return gj, gk
