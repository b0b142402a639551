"""Pin the Rys oracle (oracle/rys.py), the groundwork of a Rys VRR for the
large classes: its rule against the reference's own fp64 nodes and weights
(rys/roots.py roots_weights, n = 1..5, T from 0 to 1e4 across the
reference's switch) to 1e-13 relative and against the Boys moments
(n to 7, (ff|ff)'s count) to 1e-13; its ERI blocks against the MMD oracle on
random quartets of a cluster with shells to l = 3 to 1e-13 of the block."""

import numpy as np
import pytest

from conftest import golden


def test_rule_matches_reference():
    from oracle import rys
    z = golden("rys_roots.npz")
    for n in range(1, 6):
        for k, T in enumerate(z["T"]):
            x, w = rys.roots_weights(n, T)
            xr, wr = z["x"][n - 1, k, :n], z["w"][n - 1, k, :n]
            assert np.abs(x - xr).max() <= 1e-13 * np.abs(xr).max()
            assert np.abs(w - wr).max() <= 1e-13 * np.abs(wr).max()


@pytest.mark.parametrize("n", range(1, 8))
def test_rule_reproduces_boys_moments(oracle_lib, n):
    from oracle import oracle, rys
    for T in (0.0, 0.3, 2.0, 17.0, 63.9, 64.1, 150.0, 1e4):
        x, w = rys.roots_weights(n, T)
        for m in range(2 * n):
            F = oracle.boys(m, T)
            assert abs(float((w * x ** m).sum()) - F) <= 1e-13 * F


def test_eri_blocks_match_mmd_oracle(oracle_lib):
    from felizjueves_b200 import configs
    from oracle import oracle, rys
    B = configs.cluster(3, 5).basis
    ob = oracle.OracleBasis.of(B)
    sh = B.shells
    rng = np.random.default_rng(0)
    quartets = [[int(v) for v in rng.integers(0, len(sh), 4)] for _ in range(30)]
    fs = [i for i, s in enumerate(sh) if s.l == 3][:2]
    quartets.append([fs[0], fs[1], fs[0], fs[1]])  # (ff|ff): seven roots
    for q in quartets:
        r = rys.eri_block(*[sh[i] for i in q])
        m = oracle.eri_block(ob, *q).reshape(r.shape)
        assert np.abs(r - m).max() <= 1e-13 * np.abs(m).max(), q
