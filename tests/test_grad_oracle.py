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
