"""CPU oracle of the fused build's six-block screen (TEST INFRASTRUCTURE
ONLY: tests/ import it; the product never does).

Restates the reference's prediction of which launched quartets the F kernel
skips (eri/fock/walk_f.py:344-353, `six_block`; the rule as
eri/fock/kernel_f.py:152-160 states it):

    dmax  = max over the six blocks (ab, cd, ac, ad, bc, bd) of |w| Dsh_uv,
            |w| = 2 on ab and cd (Coulomb), 1/2 on the other four (exchange)
    skip  = G_ab * (G_cd * dmax) < tau

with Dsh the largest |D| over each shell block (kernel_f.py:608-617,
`density_blocks`) and the block order of eri/fock/levers/seams.py:179.  The
weights are powers of two, so each |w| Dsh is exact and the maximum does not
depend on the order it is taken in; the bound keeps the reference's
association G_ab (G_cd dmax).  Evaluated in numpy FP64 over arrays of
quartets.
"""

from __future__ import annotations

import numpy as np

# (u, v) index pairs into the quartet (a, b, c, d), and |w| of each block
BLOCKS = ((0, 1), (2, 3), (0, 2), (0, 3), (1, 2), (1, 3))
ABS_WEIGHTS = (2.0, 2.0, 0.5, 0.5, 0.5, 0.5)


def density_blocks(D: np.ndarray, offsets, sizes) -> np.ndarray:
    """n_sh x n_sh: the largest |D| over each shell block."""
    n = len(offsets)
    A = np.abs(np.asarray(D, np.float64))
    out = np.empty((n, n))
    for s in range(n):
        rs = A[offsets[s]:offsets[s] + sizes[s]]
        for t in range(n):
            out[s, t] = rs[:, offsets[t]:offsets[t] + sizes[t]].max()
    return out


def six_block_skip(Dsh: np.ndarray, shells: np.ndarray, G_bra: np.ndarray, G_ket: np.ndarray,
                   tau: float) -> np.ndarray:
    """Skip decisions (bool) of quartets `shells` (n x 4: a, b, c, d as the
    launch orders them) with pair bounds G_bra = G_ab and G_ket = G_cd."""
    s = np.asarray(shells, np.int64)
    dmax = ABS_WEIGHTS[0] * Dsh[s[:, 0], s[:, 1]]
    for w, (u, v) in zip(ABS_WEIGHTS[1:], BLOCKS[1:]):
        t = w * Dsh[s[:, u], s[:, v]]
        dmax = np.where(dmax < t, t, dmax)
    return np.asarray(G_bra, np.float64) * (np.asarray(G_ket, np.float64) * dmax) < tau
