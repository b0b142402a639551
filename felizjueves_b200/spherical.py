"""Spherical AOs around the Cartesian G build.

    harmonics(l) -> C        (2l+1) x ncart(l): row m (-l..l) over cartesians(l)
    transform(basis) -> T    n_cart x n_sph, block diagonal, T[cart, sph]
    SphericalFock            J, K, G in real solid harmonics from a spherical D

Every kernel here is Cartesian (the reference's AOs are Cartesian; its
spherical forms are the density-fitting outputs of eri/density_fit/
kernel_eri3.py).  A spherical basis is its Cartesian one contracted by the
real solid harmonics: D_cart = T D_sph T^T, G_sph = T^T G_cart T (two GEMMs
a side on the device).

The convention is the reference's (kernel_eri3.py's spherical-output
section; PySCF / libcint order m = -l..l): s and p are the identity (p stays
x, y, z); from d up, column m is the real solid harmonic S_lm, expanded by
the closed form of Helgaker, Jorgensen and Olsen, Molecular Electronic-
Structure Theory, eqs. 6.4.47-6.4.50,

    S_lm = N_lm sum_t sum_u sum_v C^lm_tuv x^(2t+|m|-2(u+v)) y^(2(u+v)) z^(l-2t-|m|),
    C^lm_tuv = (-1)^(t+v-v_m) (1/4)^t binom(l,t) binom(l-t,|m|+t) binom(t,u) binom(|m|,2v),

v_m = 0 (m >= 0, the cosine branch) or 1/2 (m < 0, the sine branch),
normalised under the Gaussian-moment product <x^a, x^b> = prod_d (a_d + b_d
- 1)!! and then scaled by sqrt((2l-1)!!), so that an AO normalised as its
(l, 0, 0) component maps to a normalised spherical function.
"""

from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .shell import Basis, cartesians


def _odd_df(n: int) -> int:
    """n!! for odd n >= -1 ((-1)!! = 1)."""
    out = 1
    while n > 1:
        out *= n
        n -= 2
    return out


def _moment(p, q) -> int:
    s = [a + b for a, b in zip(p, q)]
    if any(x % 2 for x in s):
        return 0
    return math.prod(_odd_df(x - 1) for x in s)


@lru_cache(maxsize=None)
def _harmonics(l: int) -> tuple[tuple[float, ...], ...]:  # noqa: E741
    carts = cartesians(l)
    n = len(carts)
    if l <= 1:
        return tuple(tuple(1.0 if i == j else 0.0 for j in range(n)) for i in range(n))
    index = {c: k for k, c in enumerate(carts)}
    rows = []
    for m in range(-l, l + 1):
        am = abs(m)
        half = m < 0  # v runs over half-integers on the sine branch
        col = [0.0] * n
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                # 2v = v2 in {0, 2, 4, ...} (cosine) or {1, 3, ...} (sine), 2v <= |m|
                for v2 in range(1 if half else 0, am + 1, 2):
                    px = 2 * t + am - 2 * u - v2
                    py = 2 * u + v2
                    pz = l - 2 * t - am
                    if px < 0 or pz < 0:
                        continue
                    vm2 = 1 if half else 0
                    sign = -1.0 if (t + (v2 - vm2) // 2) % 2 else 1.0
                    c = sign * 0.25 ** t * math.comb(l, t) * math.comb(l - t, am + t) * math.comb(t, u) \
                        * math.comb(am, v2)
                    col[index[(px, py, pz)]] += c
        norm2 = sum(col[i] * col[j] * _moment(carts[i], carts[j])
                    for i in range(n) for j in range(n) if col[i] and col[j])
        k = math.sqrt(_odd_df(2 * l - 1)) / math.sqrt(norm2)
        rows.append(tuple(c * k for c in col))
    return tuple(rows)


def harmonics(l: int) -> np.ndarray:  # noqa: E741
    """Row m + l: the coefficients of S_lm over cartesians(l)."""
    if type(l) is not int or l < 0:
        raise ValueError(f"l = {l!r} is not an int >= 0")
    return np.array(_harmonics(l))


def n_spherical(basis: Basis) -> int:
    return sum(2 * s.l + 1 for s in basis.shells)


def transform(basis: Basis) -> np.ndarray:
    """T (n_cart x n_sph): shell k's block harmonics(l_k)^T at its Cartesian
    and spherical offsets."""
    T = np.zeros((basis.n_ao, n_spherical(basis)))
    j = 0
    for s, off in zip(basis.shells, basis.offsets):
        h = harmonics(s.l)
        T[off:off + s.n_cart, j:j + 2 * s.l + 1] = h.T
        j += 2 * s.l + 1
    return T


class SphericalFock:
    """J, K, G of a spherical density through the Cartesian engine:
    D_cart = T D_sph T^T (made exactly symmetric, as the plan requires),
    then G_sph = T^T G_cart T, on the device."""

    def __init__(self, basis: Basis, device: int = 0):
        import torch

        from .fock import FockEngine
        self.eng = FockEngine(basis, device)
        self.T = torch.tensor(transform(basis), device=f"cuda:{device}")
        self.n = self.T.shape[1]

    def _cart(self, D):
        Dc = self.T @ D @ self.T.T
        return 0.5 * (Dc + Dc.T)

    def plan(self, D_sph, tau: float = 1e-12, n: int = 4):
        import torch
        D = torch.as_tensor(np.ascontiguousarray(D_sph, np.float64), device=self.T.device)
        return self.eng.plan(self._cart(D).cpu().numpy(), tau, n)

    def build(self, D_sph, **kw):
        """(J, K, G) in the spherical AOs of the symmetric spherical D_sph
        (a cuda float64 tensor); `kw` as FockEngine.build."""
        if tuple(D_sph.shape) != (self.n, self.n):
            raise ValueError(f"D must be ({self.n}, {self.n}) in the spherical AOs")
        Dc = self._cart(D_sph).contiguous()
        J, K, G = self.eng.build(Dc, **kw)
        return tuple(self.T.T @ M @ self.T for M in (J, K, G))
