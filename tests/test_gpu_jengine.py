"""The McMurchie-Davidson J-engine (fjb_coulomb) against the reference's own
J (coulomb_matrix at tau = 0: tests/golden/jk_*.npz), the C oracle, libcint
and the fused HGP build's J; and its screened sweep against the unscreened
one within the reference's error claim |J(tau) - J(0)| <= tau * scale
(eri/j_coulomb/j.py:80-90)."""

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

from conftest import golden

pytestmark = pytest.mark.gpu

FP64_ABS = 1e-11


def _j(basis, D, tau, cuda):
    import torch
    eng = FockEngine(basis)
    Dt = torch.tensor(D, device=cuda)
    J = eng.coulomb(Dt, tau=tau)
    torch.cuda.synchronize()
    return eng, J.cpu().numpy()


@pytest.mark.parametrize("name,atoms,wfn", [("c0_1at", 1, "c0"), ("c0_2at", 2, "c0"),
                                            ("c1_1at", 1, "c1")])
def test_j_engine_matches_reference_coulomb_matrix(cuda, lib_built, name, atoms, wfn):
    w = configs.sub_workload(getattr(configs, wfn)(), atoms)
    g = golden(f"jk_{name}.npz")
    _, J = _j(w.basis, w.D, 0.0, cuda)
    assert np.abs(J - g["J"]).max() <= FP64_ABS
    assert np.array_equal(J, J.T)  # one writer per element, mirrored


@pytest.mark.parametrize("atoms,seed", [(3, 5), (4, 7)])
def test_j_engine_matches_oracle_every_class(cuda, lib_built, oracle_lib, atoms, seed):
    """Every (bra L, ket L) class to (6, 6) at once, unscreened."""
    w = configs.cluster(atoms, seed)
    _, J = _j(w.basis, w.D, 0.0, cuda)
    Jo, _ = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(J - Jo).max() <= FP64_ABS


def test_j_engine_matches_libcint(cuda, lib_built):
    from test_gpu_fock import _basis_from_npz
    for name in ("h2o_ccpvdz", "co_ccpvtz"):
        g = golden(f"libcint_{name}.npz")
        _, J = _j(_basis_from_npz(g), g["D"], 0.0, cuda)
        assert np.abs(J - g["vj"]).max() <= 1e-12 * np.abs(g["vj"]).max()


def test_j_engine_screened_and_fused_build(cuda, lib_built):
    """At tau = 1e-12 the sorted break drops terms within the error claim;
    the result equals the fused HGP build's J at the same tau."""
    import torch
    w = configs.cluster(8, 11)
    eng, J0 = _j(w.basis, w.D, 0.0, cuda)
    Dt = torch.tensor(w.D, device=cuda)
    Jt = eng.coulomb(Dt, tau=w.tau).cpu().numpy()
    eng.plan(w.D, w.tau, w.n_mag)
    Jf = eng.build(Dt)[0].cpu().numpy()
    d_scr = float(np.abs(Jt - J0).max())
    d_fused = float(np.abs(Jt - Jf).max())
    print(f"J-engine: screened vs unscreened {d_scr:.2e}, vs fused build {d_fused:.2e}, "
          f"{eng.j_launches()} launches")
    assert d_scr <= 1e-10
    assert d_fused <= 1e-10


@pytest.mark.parametrize("atoms,seed", [(3, 5), (6, 11)])
def test_j_engine_fp32_tier(cuda, lib_built, oracle_lib, atoms, seed):
    """The FP32 E/R tier (fjb_coulomb_mixed) at the 1e-9 routing bound:
    within the metric's 1e-8 budget of the FP64 J-engine and of the oracle;
    a bound above every key runs every chunk in FP32, at FP32 accuracy."""
    import torch
    w = configs.cluster(atoms, seed)
    eng = FockEngine(w.basis)
    D = torch.tensor(w.D, device=cuda)
    J64 = eng.coulomb(D, tau=0.0).clone()
    J32 = eng.coulomb(D, tau=0.0, threshold=1e-9).clone()
    Jall = eng.coulomb(D, tau=0.0, threshold=1e30).clone()
    torch.cuda.synchronize()
    Jo, _ = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    d64 = float((J32 - J64).abs().max())
    dor = float(np.abs(J32.cpu().numpy() - Jo).max())
    dall = float((Jall - J64).abs().max() / J64.abs().max())
    print(f"{atoms} atoms: mixed vs FP64 {d64:.2e}, vs oracle {dor:.2e}; all-FP32 relative {dall:.2e}")
    assert d64 <= 1e-8 and dor <= 1e-8
    assert 0.0 < dall <= 1e-5
