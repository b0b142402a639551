"""The SCF driver's loop (felizjueves_b200/scf.py) on CPU with the oracle as
its injected evaluators: converged orbital energies and density against
PySCF's converged RHF recorded in the reference's fixtures (conv_tol 1e-12);
incremental (difference-density) and full G builds reach the same result."""

import numpy as np
import pytest

from conftest import golden
from test_onee_oracle import basis_of, nuclei_of


class OracleBuilders:
    def __init__(self, basis):
        from oracle import oracle
        self.basis = basis
        self.ob = oracle.OracleBasis.of(basis)
        self.oracle = oracle

    def one_electron(self, nuclei):
        import torch
        from oracle import one_electron
        S, T, V = one_electron.matrices(self.basis, nuclei)
        return torch.tensor(S), torch.tensor(T + V)

    def g(self, D):
        import torch
        J, K = self.oracle.jk(self.ob, D.numpy())
        return torch.tensor(J - 0.5 * K)


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631g"])
@pytest.mark.parametrize("incremental", [True, False])
def test_scf_loop_matches_pyscf(oracle_lib, name, incremental):
    from felizjueves_b200.scf import rhf
    g = golden(f"scf_{name}.npz")
    B = basis_of(g)
    r = rhf(B, nuclei_of(g), builders=OracleBuilders(B), incremental=incremental,
            e_tol=1e-11, d_tol=1e-9)
    assert r.converged
    assert np.abs(r.mo_energy - g["mo_energy"]).max() <= 1e-7
    assert np.abs(r.D - g["D"]).max() <= 1e-6
    kinds = {h[2] for h in r.history}
    assert kinds == ({"full", "delta"} if incremental else {"full"})


def test_scf_refusals():
    from felizjueves_b200.scf import nuclear_repulsion, rhf
    g = golden("scf_h2o_sto3g.npz")
    B = basis_of(g)
    with pytest.raises(ValueError, match="even"):
        rhf(B, nuclei_of(g), n_elec=9, builders=object())
    with pytest.raises(ValueError, match="coincide"):
        nuclear_repulsion([(1.0, (0.0, 0.0, 0.0)), (1.0, (0.0, 0.0, 0.0))])
