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
