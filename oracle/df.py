"""Density-fitting oracle (TEST INFRASTRUCTURE ONLY): (P|Q) and (mn|P) from
the C oracle's eri_block with every aux primitive paired with a unit s
function (exponent 0, coefficient 1) -- the reference's aux dressing
c (pi/alpha)^{3/2} (eri/density_fit/metric.py:1-60) -- and DF-J/K in numpy
FP64 with the metric's Cholesky factor.  The reference computes no DF-J/K,
so that part restates the standard formula (parity unpinned); the integrals
are pinned to libcint's by tests/test_oracle.py."""

from __future__ import annotations

import numpy as np

from . import oracle as O


def _combined(ao, aux):
    """One oracle basis: the AO shells (if any), the aux shells, the unit."""
    parts = ([ao.flat()] if ao is not None else []) + [aux.flat()]
    l, c, p0, npr, ex, co = [], [], [], [], [], []
    for p in parts:
        base = len(ex)
        l += list(p["l"]); c += list(p["centre"]); p0 += [base + x for x in p["prim0"]]
        npr += list(p["nprim"]); ex += list(p["exps"]); co += list(p["coefs"])
    l.append(0); c.append(np.zeros(3)); p0.append(len(ex)); npr.append(1)
    ex.append(0.0); co.append(1.0)
    return O.OracleBasis(np.array(l), np.array(c), np.array(p0), np.array(npr),
                         np.array(ex), np.array(co))


def metric(aux) -> np.ndarray:
    ob = _combined(None, aux)
    ns = len(aux.shells)
    unit = ns
    V = np.zeros((aux.n_ao, aux.n_ao))
    for P in range(ns):
        for Q in range(P, ns):
            nP, nQ = aux.shells[P].n_cart, aux.shells[Q].n_cart
            blk = O.eri_block(ob, P, unit, Q, unit).reshape(nP, nQ)
            oP, oQ = aux.offsets[P], aux.offsets[Q]
            V[oP:oP + nP, oQ:oQ + nQ] = blk
            V[oQ:oQ + nQ, oP:oP + nP] = blk.T
    return V


def eri3(ao, aux) -> np.ndarray:
    ob = _combined(ao, aux)
    na, nx = len(ao.shells), len(aux.shells)
    unit = na + nx
    T = np.zeros((ao.n_ao, ao.n_ao, aux.n_ao))
    for a in range(na):
        for b in range(a, na):
            for P in range(nx):
                sa, sb, sp = ao.shells[a].n_cart, ao.shells[b].n_cart, aux.shells[P].n_cart
                blk = O.eri_block(ob, a, b, na + P, unit).reshape(sa, sb, sp)
                oa, ob_, op = ao.offsets[a], ao.offsets[b], aux.offsets[P]
                T[oa:oa + sa, ob_:ob_ + sb, op:op + sp] = blk
                T[ob_:ob_ + sb, oa:oa + sa, op:op + sp] = blk.transpose(1, 0, 2)
    return T


def df_jk(ao, aux, D):
    V = metric(aux)
    T = eri3(ao, aux)
    L = np.linalg.cholesky(V)
    n, nx = ao.n_ao, aux.n_ao
    B = np.linalg.solve(L, T.reshape(n * n, nx).T).reshape(nx, n, n)
    gamma = np.einsum("pmn,mn->p", B, D)
    J = np.einsum("pmn,p->mn", B, gamma)
    K = np.einsum("pml,ls,pns->mn", B, D, B, optimize=True)
    return J, K
