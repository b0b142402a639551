"""Pin the nuclear-gradient oracle (oracle/gradient.py): the derivative
J and K matrices vj1, vk1 and the per-atom J and K gradient terms against
PySCF's grad.rhf.get_jk over libcint's int2e_ip1, as recorded in the
reference's gradient fixtures (H2O STO-3G / 6-31G / cc-pVDZ, NH2F 6-31G).
Bars: 1e-13 of the largest element; the per-atom terms 1e-12 absolute."""

import numpy as np
import pytest

from conftest import golden
from test_onee_oracle import basis_of

CASES = ["h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "nh2f_631g"]


@pytest.mark.parametrize("name", CASES)
def test_gradient_jk_matches_pyscf(oracle_lib, name):
    from oracle import gradient
    s = golden(f"scf_{name}.npz")
    g = golden(f"grad_{name}.npz")
    D = g["density"]
    vj1, vk1 = gradient.jk_derivatives(basis_of(s), D)
    for got, ref in ((vj1, g["vj1"]), (vk1, g["vk1"])):
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    gj, gk = gradient.gradient_jk(vj1, vk1, D, g["ao_atom"], len(s["charges"]))
    assert np.abs(gj - g["grad_j"]).max() <= 1e-12
    assert np.abs(gk - g["grad_k"]).max() <= 1e-12


@pytest.mark.parametrize("name", CASES)
def test_shift_assembly_with_oracle_jk(oracle_lib, name):
    """The product's assembly (felizjueves_b200/gradient.py: the extended
    basis, one J/K build over it, the shift combination) with the oracle's
    J/K as the injected evaluator reproduces PySCF's vj1, vk1 and terms."""
    from felizjueves_b200 import gradient
    from oracle import oracle
    s = golden(f"scf_{name}.npz")
    g = golden(f"grad_{name}.npz")
    D = g["density"]
    B = basis_of(s)
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]

    def jk(Bx, Dx):
        return oracle.jk(oracle.OracleBasis.of(Bx), Dx)

    vj1, vk1 = gradient.jk_derivatives(B, D, jk=jk)
    for got, ref in ((vj1, g["vj1"]), (vk1, g["vk1"])):
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.array_equal(gradient.ao_atoms(B, nuclei), g["ao_atom"])
    gj, gk = gradient.gradient_jk(B, D, nuclei, jk=jk)
    assert np.abs(gj - g["grad_j"]).max() <= 1e-12 and np.abs(gk - g["grad_k"]).max() <= 1e-12


def test_extended_basis_refuses_f():
    from felizjueves_b200 import gradient
    from felizjueves_b200.shell import Basis, Shell
    with pytest.raises(ValueError, match="l = 2"):
        gradient.extended_basis(Basis((Shell(3, (0.0, 0.0, 0.0), [1.0], [1.0]),)))


@pytest.mark.parametrize("name", CASES)
def test_rhf_gradient_assembly_with_oracle(oracle_lib, name):
    """The product's whole RHF gradient (felizjueves_b200/gradient.py
    rhf_gradient) with the oracle's one-electron matrices and J/K injected:
    libcint's int1e_ipovlp / ipkin / ipnuc / iprinv (1e-13 of the largest
    element) and PySCF's per-atom h, S, J, K, nuclear terms and total
    (1e-11)."""
    from felizjueves_b200 import gradient
    from oracle import one_electron, oracle
    s = golden(f"scf_{name}.npz")
    g = golden(f"grad_{name}.npz")
    B = basis_of(s)
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]

    def onee(Bx, nuc):
        return one_electron.matrices(Bx, nuc)

    def jk(Bx, Dx):
        return oracle.jk(oracle.OracleBasis.of(Bx), Dx)

    ip = gradient.one_electron_derivatives(B, nuclei, onee=onee)
    for got, key in zip(ip, ("int1e_ipovlp", "int1e_ipkin", "int1e_ipnuc", "int1e_iprinv")):
        assert np.abs(got - g[key]).max() <= 1e-13 * np.abs(g[key]).max(), key
    r = gradient.rhf_gradient(B, nuclei, g["density"], g["dme"], jk=jk, onee=onee)
    for term in ("h", "s", "j", "k", "nuc", "total"):
        assert np.abs(r[term] - g[f"grad_{term}"]).max() <= 1e-11, term


def test_scf_then_gradient_with_oracle(oracle_lib):
    """The SCF loop and the gradient assembly chained, the oracle injected
    into both: PySCF's total gradient within 1e-7 (measured 4.6e-9)."""
    from felizjueves_b200 import gradient
    from felizjueves_b200.scf import rhf
    from oracle import one_electron, oracle
    from test_scf import OracleBuilders
    s = golden("scf_h2o_631g.npz")
    g = golden("grad_h2o_631g.npz")
    B = basis_of(s)
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]
    r = rhf(B, nuclei, builders=OracleBuilders(B), e_tol=1e-11, d_tol=1e-9)
    C = r.mo_coeff[:, :5]
    W = 2.0 * (C * r.mo_energy[:5]) @ C.T
    out = gradient.rhf_gradient(B, nuclei, r.D, 0.5 * (W + W.T),
                                jk=lambda Bx, Dx: oracle.jk(oracle.OracleBasis.of(Bx), Dx),
                                onee=lambda Bx, n: one_electron.matrices(Bx, n))
    assert np.abs(out["total"] - g["grad_total"]).max() <= 1e-7


@pytest.mark.parametrize("entry,case,bse", [("jx1_h2o_sto3g_bse", "h2o_sto3g_j", "sto-3g.json"),
                                            ("jx1_h2o_ccpvdz_bse", "h2o_ccpvdz_j", "cc-pVDZ.json")])
def test_vj1_of_bse_documents_matches_pyscf(oracle_lib, entry, case, bse):
    """vj1 (grad.rhf.get_jk's Coulomb derivative matrices) over a BSE
    document read as it stands (no free-primitive reduction), against
    PySCF's over the same document (the reference's numerical golden store,
    test/golden/numeric/jx1_*_bse.npy): 1e-12 of max|vj1|."""
    import json
    import os
    from conftest import GOLDEN
    from felizjueves_b200 import basis_io
    from oracle import gradient
    with open(os.path.join(GOLDEN, "bse_subset.json")) as fh:
        doc = json.load(fh)["sets"][bse]
    g1 = golden(f"onee_{case}.npz")
    atoms = [(z, tuple(c)) for z, c in zip(g1["charges"], g1["coords"])]
    B = basis_io.from_bse(basis_io.parse(doc), atoms, reduce=False)
    g = golden(f"numeric_{entry}.npz")
    vj1, _ = gradient.jk_derivatives(B, g["D"])
    assert np.abs(vj1 - g["J"]).max() <= 1e-12 * np.abs(g["J"]).max()
