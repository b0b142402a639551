"""The J and K terms of the nuclear gradient on the GPU
(felizjueves_b200/gradient.py: one build over the shift-extended basis)
against PySCF's grad.rhf.get_jk over libcint's int2e_ip1, as recorded in
the reference's gradient fixtures: vj1, vk1 to 1e-12 of the largest
element, the per-atom J and K terms to 1e-10."""

import numpy as np
import pytest

from conftest import golden
from test_onee_oracle import basis_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "nh2f_631g"])
def test_gradient_jk_matches_pyscf(cuda, lib_built, name):
    from felizjueves_b200 import gradient
    s = golden(f"scf_{name}.npz")
    g = golden(f"grad_{name}.npz")
    D = g["density"]
    B = basis_of(s)
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]
    vj1, vk1 = gradient.jk_derivatives(B, D)
    for got, ref in ((vj1, g["vj1"]), (vk1, g["vk1"])):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    gj, gk = gradient.gradient_jk(B, D, nuclei)
    assert np.abs(gj - g["grad_j"]).max() <= 1e-10 and np.abs(gk - g["grad_k"]).max() <= 1e-10


@pytest.mark.parametrize("name", ["h2o_631g", "nh2f_631g"])
def test_rhf_gradient_matches_pyscf(cuda, lib_built, name):
    """The whole RHF nuclear gradient on the GPU (one-electron derivative
    matrices and J/K terms from shift-extended builds): every term and the
    total against PySCF's at the recorded density, to 1e-10."""
    from felizjueves_b200 import gradient
    s = golden(f"scf_{name}.npz")
    g = golden(f"grad_{name}.npz")
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]
    r = gradient.rhf_gradient(basis_of(s), nuclei, g["density"], g["dme"])
    for term in ("h", "s", "j", "k", "nuc", "total"):
        assert np.abs(r[term] - g[f"grad_{term}"]).max() <= 1e-10, term


def test_scf_then_gradient(cuda, lib_built):
    """SCF to convergence, then the gradient from its own D and W: PySCF's
    total gradient within 1e-6 (the two converged densities differ by ~1e-8,
    and the gradient is not variational in D)."""
    from felizjueves_b200 import gradient
    from felizjueves_b200.scf import rhf
    s = golden("scf_h2o_631g.npz")
    g = golden("grad_h2o_631g.npz")
    B = basis_of(s)
    nuclei = [(float(z), tuple(c)) for z, c in zip(s["charges"], s["coords"])]
    r = rhf(B, nuclei, e_tol=1e-11, d_tol=1e-9)
    occ = 5
    C = r.mo_coeff[:, :occ]
    W = 2.0 * (C * r.mo_energy[:occ]) @ C.T
    W = 0.5 * (W + W.T)
    out = gradient.rhf_gradient(B, nuclei, r.D, W)
    assert np.abs(out["total"] - g["grad_total"]).max() <= 1e-6
