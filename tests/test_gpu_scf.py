"""The SCF driver on the GPU (felizjueves_b200/scf.py with the sm_100a
one-electron and G builds): converged orbital energies within 1e-7 and the
density within 1e-6 of PySCF's converged RHF in the reference's fixtures;
the incremental loop (difference-density builds between full ones) and
the routed (mixed-precision) G reach the same result."""

import numpy as np
import pytest

from conftest import golden
from test_onee_oracle import basis_of, nuclei_of

pytestmark = pytest.mark.gpu

CASES = ["h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "nh2f_631g"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("incremental", [True, False])
def test_gpu_scf_matches_pyscf(cuda, lib_built, name, incremental):
    from felizjueves_b200.scf import GpuBuilders, rhf
    g = golden(f"scf_{name}.npz")
    B = basis_of(g)
    b = GpuBuilders(B, tau=1e-12)
    r = rhf(B, nuclei_of(g), builders=b, incremental=incremental, e_tol=1e-11, d_tol=1e-9)
    assert r.converged, r.history[-3:]
    de = float(np.abs(r.mo_energy - g["mo_energy"]).max())
    dd = float(np.abs(r.D - g["D"]).max())
    print(f"{name} incremental={incremental}: {r.iterations} iterations, E = {r.energy:.10f}, "
          f"max|de| {de:.2e}, max|dD| {dd:.2e}, computed quartets per build {b.computed}")
    assert de <= 1e-7 and dd <= 1e-6
    if incremental:
        # both kinds of build ran; the quartet counts are printed, not held:
        # at these sizes |dD| ~ 1e-9 still leaves almost every quartet above
        # tau, and a plan of dD bins its pairs by dD's own magnitudes, so a
        # difference build can compute a few more quartets than a full one
        assert {h[2] for h in r.history} == {"full", "delta"}


def test_gpu_scf_routed(cuda, lib_built):
    from felizjueves_b200 import _lib
    from felizjueves_b200.scf import rhf
    g = golden("scf_h2o_ccpvdz.npz")
    r = rhf(basis_of(g), nuclei_of(g), precision=_lib.FJB_ROUTED, threshold=1e-9, e_tol=1e-11, d_tol=1e-9)
    assert r.converged
    assert np.abs(r.mo_energy - g["mo_energy"]).max() <= 1e-7
