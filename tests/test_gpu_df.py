"""Density fitting on the GPU: (P|Q) and (mn|P) from the HGP kernels against
libcint's (the reference's fixtures), and DF-J/K against the oracle's numpy
restatement (FP64: max(1e-10, 1e-15 cond(V)) of max|.|, the metric solve
amplifying integral rounding by its condition number; the library's
fjb_df_jk: J in FP64 (1e-12 of max|J| against the FP64 contractions), K on
the tensor cores as a BF16x3 split (error reported, bounded by 1e-5 of
max|K|)).
DF's own error against the exact
4-centre J, K is reported (it is the fitting error, not a kernel error)."""

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs

pytestmark = pytest.mark.gpu


def _df_bases(z):
    from felizjueves_b200.shell import Basis, Shell

    def mk(prefix):
        out = []
        for s in range(len(z[prefix + "l"])):
            p0, n = int(z[prefix + "prim0"][s]), int(z[prefix + "nprim"][s])
            out.append(Shell(int(z[prefix + "l"][s]), tuple(z[prefix + "centre"][s]),
                             z[prefix + "exps"][p0:p0 + n], z[prefix + "coefs"][p0:p0 + n]))
        return Basis(tuple(out))
    return mk("ao_"), mk("aux_")


@pytest.mark.parametrize("name", ["prim_spd_f_auxi_metric", "h2o_ccpvtz_jkfit_metric",
                                  "prim_spd_f_auxi_3c", "h2o_sto3g_jkfit_3c"])
def test_df_integrals_match_libcint(cuda, lib_built, name):
    from felizjueves_b200.df import DFEngine
    z = golden(f"df_{name}.npz")
    ao, aux = _df_bases(z)
    eng = DFEngine(ao, aux)
    got = (eng.metric() if str(z["kind"]) == "metric" else eng.eri3()).cpu().numpy()
    ref = z["value"]
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print(f"{name}: max rel {err:.2e}")
    assert err <= 1e-12


def test_df_jk_matches_oracle(cuda, lib_built, oracle_lib):
    import torch
    from felizjueves_b200.df import DFEngine
    from oracle import df as odf
    w = configs.cluster(2, 3)
    aux = configs.aux_basis(w)
    eng = DFEngine(w.basis, aux)
    D = torch.tensor(w.D, device=cuda)
    B = eng.factors()
    J, K = eng.jk(D, "fp64", B=B)
    Jo, Ko = odf.df_jk(w.basis, aux, w.D)
    sJ, sK = np.abs(Jo).max(), np.abs(Ko).max()
    # The fit solves with the metric, so two FP64 paths whose integrals agree
    # to ~1e-14 differ by up to cond(V) times that: the bar scales with it.
    cond = float(np.linalg.cond(odf.metric(aux)))
    tol = max(1e-10, 1e-15 * cond)
    dJ = np.abs(J.cpu().numpy() - Jo).max() / sJ
    dK = np.abs(K.cpu().numpy() - Ko).max() / sK
    print(f"cond(V) {cond:.2e}; fp64 DF vs oracle: J {dJ:.2e} K {dK:.2e} (bar {tol:.1e})")
    assert dJ <= tol and dK <= tol
    J3, K3 = eng.jk(D, "bf16x3", B=B)
    eJ = float((J3 - J).abs().max()) / sJ
    eK = float((K3 - K).abs().max()) / sK
    Je, Ke = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    fJ = np.abs(J.cpu().numpy() - Je).max() / np.abs(Je).max()
    fK = np.abs(K.cpu().numpy() - Ke).max() / np.abs(Ke).max()
    print(f"bf16x3 vs fp64 DF: J {eJ:.2e} K {eK:.2e}; DF vs exact: J {fJ:.2e} K {fK:.2e}")
    # J is FP64 on both paths; K's FP32-level products (2^-24) summed with
    # cancellation over aux x AO signed terms keep ~1e-6, orders below the
    # fitting error of this aux recipe (DF vs exact above).
    assert eJ <= 1e-12 and eK <= 1e-5
    assert eK < 1e-2 * fK


def test_df_tensor_core_k_over_tiles(cuda, lib_built):
    """fjb_df_jk on a 5-atom cluster (155 AO: two 128-wide output tiles with
    a ragged edge; 450 aux functions: 1,090 K-tiles in the second GEMM),
    against the FP64 contractions of the same factors."""
    import torch
    from felizjueves_b200.df import DFEngine
    w = configs.cluster(5, 9)
    aux = configs.aux_basis(w)
    eng = DFEngine(w.basis, aux)
    D = torch.tensor(w.D, device=cuda)
    B = eng.factors()
    J, K = eng.jk(D, "fp64", B=B)
    J3, K3 = eng.jk(D, "bf16x3", B=B)
    eJ = float((J3 - J).abs().max() / J.abs().max())
    eK = float((K3 - K).abs().max() / K.abs().max())
    print(f"n_ao {w.n_ao} n_aux {aux.n_ao}: J {eJ:.2e} K {eK:.2e}")
    assert eJ <= 1e-12 and eK <= 1e-5
    assert float((K3 - K3.T).abs().max()) <= 1e-5 * float(K.abs().max())
