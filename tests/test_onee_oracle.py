"""Pin the one-electron oracle (oracle/one_electron.py): S, T, V and
h = T + V against the libcint int1e_ovlp / int1e_kin / int1e_nuc / hcore
fixtures the reference tracks, and against the reference's own
overlap_matrix / kinetic_matrix / potential_matrix on a seeded cluster with
shells to l = 3.  Bar: 1e-12 of the matrix's largest element (the
reference's libcint tolerance for one-electron matrices)."""

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200.shell import Basis, Shell

FIXTURES = ["h2_sto3g_j", "h2o_sto3g_j", "h2o_631g_j", "h2o_ccpvdz_j", "h10_chain_ccpvdz_j",
            "hf_ccpvtz", "prim_spd_f", "prim_spdf", "co_ccpvtz"]


def basis_of(g):
    shells = []
    for s in range(len(g["l"])):
        p0, n = int(g["prim0"][s]), int(g["nprim"][s])
        shells.append(Shell(int(g["l"][s]), tuple(g["centre"][s]), g["exps"][p0:p0 + n],
                            g["coefs"][p0:p0 + n]))
    return Basis(tuple(shells))


def nuclei_of(g):
    return [(float(z), tuple(c)) for z, c in zip(g["charges"], g["coords"])]


def _close(got, ref, rel=1e-12):
    return np.abs(got - ref).max() <= rel * np.abs(ref).max()


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_libcint(oracle_lib, name):
    from oracle import one_electron
    g = golden(f"onee_{name}.npz")
    S, T, V = one_electron.matrices(basis_of(g), nuclei_of(g))
    assert _close(S, g["S"]) and _close(T, g["T"]) and _close(V, g["V"])
    assert _close(T + V, g["H"])
    for M in (S, T, V):
        assert np.array_equal(M, M.T)


def test_oracle_matches_reference_cluster3(oracle_lib):
    from felizjueves_b200 import configs
    from oracle import one_electron
    g = golden("onee_ref_cluster3.npz")
    w = configs.cluster(3, 5)
    S, T, V = one_electron.matrices(w.basis, nuclei_of(g))
    for got, ref in ((S, g["S"]), (T, g["T"]), (V, g["V"])):
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
