"""GPU parity of the one-electron matrices (fjb_one_electron through the C
ABI): S, T, V and H = T + V against the libcint int1e_* / hcore fixtures the
reference tracks (1e-12 of the matrix's largest element), against the
reference's own overlap/kinetic/potential matrices on a seeded cluster with
shells to l = 3, and against the oracle on a 6-atom cluster (1e-13 of the
largest element).  Every matrix exactly symmetric."""

import numpy as np
import pytest

from conftest import golden
from test_onee_oracle import FIXTURES, basis_of, nuclei_of

pytestmark = pytest.mark.gpu


def _rel(got, ref):
    return float(np.abs(got - ref).max() / np.abs(ref).max())


def _gpu(basis, nuclei):
    from felizjueves_b200.fock import FockEngine
    eng = FockEngine(basis)
    return [M.cpu().numpy() for M in eng.one_electron(nuclei)]


@pytest.mark.parametrize("name", FIXTURES)
def test_one_electron_matches_libcint(cuda, lib_built, name):
    g = golden(f"onee_{name}.npz")
    S, T, V, H = _gpu(basis_of(g), nuclei_of(g))
    for got, key in ((S, "S"), (T, "T"), (V, "V"), (H, "H")):
        assert _rel(got, g[key]) <= 1e-12, (key, _rel(got, g[key]))
        assert np.array_equal(got, got.T)


def test_one_electron_matches_reference_cluster3(cuda, lib_built):
    from felizjueves_b200 import configs
    g = golden("onee_ref_cluster3.npz")
    S, T, V, H = _gpu(configs.cluster(3, 5).basis, nuclei_of(g))
    for got, key in ((S, "S"), (T, "T"), (V, "V")):
        assert _rel(got, g[key]) <= 1e-13, (key, _rel(got, g[key]))
    assert np.array_equal(H, T + V)


def test_one_electron_matches_oracle_cluster6(cuda, lib_built, oracle_lib):
    from felizjueves_b200 import configs
    from oracle import one_electron
    w = configs.cluster(6, 11)
    centres = []
    for s in w.basis.shells:
        if s.centre not in centres:
            centres.append(s.centre)
    nuclei = [(float(1 + k % 9), c) for k, c in enumerate(centres)]
    S, T, V, H = _gpu(w.basis, nuclei)
    So, To, Vo = one_electron.matrices(w.basis, nuclei)
    for got, ref in ((S, So), (T, To), (V, Vo)):
        assert _rel(got, ref) <= 1e-13
        assert np.array_equal(got, got.T)


def test_one_electron_subsets_and_no_nuclei(cuda, lib_built):
    from felizjueves_b200.fock import FockEngine, overlap_matrix
    g = golden("onee_h2o_631g_j.npz")
    B = basis_of(g)
    eng = FockEngine(B)
    S, T, V, H = eng.one_electron(nuclei_of(g), want=("V",))
    assert S is None and T is None and H is None
    assert _rel(V.cpu().numpy(), g["V"]) <= 1e-12
    # no nuclei: V = 0 exactly and H = T
    S, T, V, H = eng.one_electron([])
    assert int((V != 0).sum()) == 0 and bool((H == T).all())
    assert _rel(overlap_matrix(B), g["S"]) <= 1e-12


def test_bse_document_to_libcint_jk(cuda, lib_built):
    """A molecule read from its Basis Set Exchange document (basis_io) runs
    through the C ABI to libcint's J and K: H2O in cc-pVDZ (reduced form)."""
    import json
    import os

    from conftest import GOLDEN
    from felizjueves_b200 import basis_io
    from felizjueves_b200.fock import FockEngine
    with open(os.path.join(GOLDEN, "bse_subset.json")) as fh:
        dz = basis_io.parse(json.load(fh)["sets"]["cc-pVDZ.json"])
    g1 = golden("onee_h2o_ccpvdz_j.npz")
    g2 = golden("libcint_h2o_ccpvdz.npz")
    B = basis_io.from_bse(dz, nuclei_of(g1), reduce=True)
    eng = FockEngine(B)
    eng.plan(g2["D"], 0.0, 4)
    J, K, G = eng.build_host(g2["D"])
    assert _rel(J, g2["vj"]) <= 1e-12 and _rel(K, g2["vk"]) <= 1e-12
    S, T, V, H = [M.cpu().numpy() for M in eng.one_electron(nuclei_of(g1))]
    assert _rel(H, g1["H"]) <= 1e-12
