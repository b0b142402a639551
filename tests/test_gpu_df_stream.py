"""The streamed DF build: the three-centre Rys kernel (fjb_df_eri3) against
the oracle's (mn|P) block by block, the tensor-core Z Z^T (fjb_df_syrk)
against FP64, and DFEngine.jk_streamed against the oracle's DF-J/K
(oracle/df.py) at the FP64 bar the metric's condition number sets, for
semidefinite and indefinite densities and several aux block sizes."""

import numpy as np
import pytest

from felizjueves_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from oracle import df as odf
    w = configs.cluster(2, 5)  # cond(V) 3e9
    aux = configs.aux_basis(w)
    return w, aux, odf.eri3(w.basis, aux), odf


@pytest.mark.parametrize("block", [40, 200])
def test_eri3_kernel_matches_oracle(cuda, lib_built, small, block):
    from felizjueves_b200.df import DFEngine
    w, aux, To, _ = small
    eng = DFEngine(w.basis, aux)
    scale = np.abs(To).max()
    blocks = eng.aux_blocks(block)
    assert blocks[0][2] == 0 and blocks[-1][3] == aux.n_ao
    for s0, s1, p0, p1 in blocks:
        got = eng.eri3_block(s0, s1, tau=0.0).cpu().numpy()
        assert got.shape == (w.n_ao, w.n_ao, p1 - p0)
        err = np.abs(got - To[:, :, p0:p1]).max() / scale
        assert err <= 1e-13, (s0, s1, err)
    # screened: every dropped block is below tau by Schwarz
    got = eng.eri3_block(0, len(aux.shells), tau=1e-9).cpu().numpy()
    assert np.abs(got - To).max() <= 1e-9


def test_syrk_matches_fp64(cuda, lib_built):
    """Ragged shapes (rows not a multiple of 128, cols not of 64) and a
    contraction long enough for several FP32 partial sums."""
    import torch
    from felizjueves_b200.df import DFEngine
    w = configs.cluster(1, 3)
    eng = DFEngine(w.basis, configs.aux_basis(w))
    g = torch.Generator(device=cuda).manual_seed(5)
    for rows, cols in ((37, 100), (300, 40000)):
        Z = torch.randn((rows, cols), dtype=torch.float64, device=cuda, generator=g)
        K = eng.syrk(Z)
        R = Z @ Z.T
        err = float((K - R).abs().max() / R.abs().max())
        print(f"syrk {rows} x {cols}: max rel {err:.2e}")
        # FP32 partial sums of at most 16,384 products of 24-bit operands:
        # sqrt(16384) 2^-24 = 7.6e-6 of the largest |Z Z^T|
        assert err <= 1e-5


@pytest.mark.parametrize("perturb", [False, True])
def test_jk_streamed_matches_oracle(cuda, lib_built, oracle_lib, small, perturb):
    import torch
    from felizjueves_b200.df import DFEngine
    w, aux, _, odf = small
    Dn = configs.perturbed_density(w.D, 1, scale=1e-2) if perturb else w.D
    eng = DFEngine(w.basis, aux)
    D = torch.tensor(Dn, device=cuda)
    Jo, Ko = odf.df_jk(w.basis, aux, Dn)
    sJ, sK = np.abs(Jo).max(), np.abs(Ko).max()
    cond = float(np.linalg.cond(odf.metric(aux)))
    tol = max(1e-10, 1e-15 * cond)
    for block in (50, 1000):
        J, K = eng.jk_streamed(D, mode="fp64", block=block, tau=0.0)
        dJ = np.abs(J.cpu().numpy() - Jo).max() / sJ
        dK = np.abs(K.cpu().numpy() - Ko).max() / sK
        print(f"block {block}: streamed fp64 vs oracle J {dJ:.2e} K {dK:.2e} (bar {tol:.1e})")
        assert dJ <= tol and dK <= tol
    t = {}
    J3, K3 = eng.jk_streamed(D, mode="bf16x3", block=200, tau=1e-12, timings=t)
    eJ = float((J3 - J).abs().max()) / sJ
    eK = float((K3 - K).abs().max()) / sK
    print(f"streamed bf16x3 vs streamed fp64: J {eJ:.2e} K {eK:.2e}; {t}")
    assert (t["n_occ"][1] > 0) == perturb
    # J: FP64 on both (tau 1e-12 drops blocks below it); K: the BF16x3 split
    assert eJ <= 1e-10 and eK <= 1e-5


def test_jk_streamed_eigh_factor_matches_dense(cuda, lib_built):
    """A metric too singular for the Cholesky factor (3 atoms, cond(V)
    1e16): the canonical-orthogonalisation factor, streamed against the
    dense factors of the same metric."""
    import torch
    from felizjueves_b200.df import DFEngine
    w = configs.cluster(3, 5)
    aux = configs.aux_basis(w)
    eng = DFEngine(w.basis, aux)
    D = torch.tensor(w.D, device=cuda)
    W, L = eng.metric_factor(method="eigh")
    assert L is None and W.shape[1] < aux.n_ao
    J, K = eng.jk_streamed(D, mode="fp64", block=100, tau=0.0, factor=(W, L))
    T = eng.eri3().reshape(w.n_ao ** 2, aux.n_ao)
    B = (W.T @ T.T).reshape(-1, w.n_ao, w.n_ao)
    Jd, Kd = eng.jk(D, "fp64", B=B)
    dJ = float((J - Jd).abs().max() / Jd.abs().max())
    dK = float((K - Kd).abs().max() / Kd.abs().max())
    print(f"eigh factor ({W.shape[1]} of {aux.n_ao} kept): streamed vs dense J {dJ:.2e} K {dK:.2e}")
    assert dJ <= 1e-9 and dK <= 1e-9
