"""The Rys kernel (rys_fock.cuh): the large classes' boundary by Rys
quadrature, then the build's HRR and digest.  Held to the oracle at the
plain FP64 bar (1e-11 max-abs) on clusters with every class to (ff|ff), to
the HGP interpreter it replaces, and in FP32 (the routed path's tier) to the
FP64 build at FP32 accuracy."""

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("atoms,seed", [(3, 5), (4, 7), (2, 3)])
def test_rys_build_matches_oracle(cuda, lib_built, oracle_lib, atoms, seed):
    w = configs.cluster(atoms, seed)
    eng = FockEngine(w.basis)
    eng.plan(w.D, 0.0, 4)
    J, K, G = eng.build_host(w.D)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(J - Jo).max() <= 1e-11
    assert np.abs(K - Ko).max() <= 1e-11
    assert np.abs(G - (Jo - 0.5 * Ko)).max() <= 1e-11


def test_rys_matches_interpreter(cuda, lib_built):
    """Same plan, same density: the Rys engine against the HGP interpreter
    on a screened 6-atom cluster (contraction degrees to 9 x 9)."""
    w = configs.cluster(6, 11)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    Jr, Kr, Gr = eng.build_host(w.D)
    eng.set_rys(False)
    Ji, Ki, Gi = eng.build_host(w.D)
    eng.set_rys(True)
    for a, b in ((Jr, Ji), (Kr, Ki), (Gr, Gi)):
        assert np.abs(a - b).max() <= 1e-11


def test_rys_fp32_tier(cuda, lib_built, oracle_lib):
    """Every unit routed to FP32: the Rys kernel's FP32 tier (and the FP32
    register bodies) against the oracle at FP32 accuracy relative to G."""
    from felizjueves_b200 import _lib, router
    w = configs.cluster(3, 5)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    _, _, G32 = eng.build_host(w.D, precision=_lib.FJB_ROUTED, threshold=1e30)
    n32, n64 = router.route_stats(eng)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    Go = Jo - 0.5 * Ko
    assert n64 == 0 and n32 > 0
    assert np.abs(G32 - Go).max() / np.abs(Go).max() <= 1e-5
