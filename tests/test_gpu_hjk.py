"""The split K build (fjb_hjk_k) over the ordered pair stream: every ordered
quartet once, K[a][c] += D[b][d] (ab|cd), on the HGP interpreter.  Held to
the oracle's K at the plain FP64 bar unscreened, in ordered and canonical
mode; the device's skip decisions equal the plan's (per launch, the
quartets computed on the device are the visits the host plan keeps); the
screened K within the bound its skipped keys give."""

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

pytestmark = pytest.mark.gpu


def _kept_per_launch(eng, P):
    b = P["batches"]
    out = []
    for li, L in enumerate(P["launches"]):
        n = int(b[L[0], 4]) * int(b[L[1], 4])
        keys, skipped = eng.hjk_keys(li, n)
        out.append(int((~skipped).sum()))
    return np.array(out)


@pytest.mark.parametrize("mode", ["ordered", "canonical"])
def test_split_k_matches_oracle_unscreened(cuda, lib_built, oracle_lib, mode):
    import torch
    w = configs.cluster(2, 5)
    eng = FockEngine(w.basis)
    P = eng.hjk_plan(w.D, 0.0, mode=mode, screen="k")
    assert P["counts"]["quartets_skipped"] == 0
    D = torch.tensor(w.D, device=cuda)
    K = eng.hjk_k(D).cpu().numpy()
    _, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    err = np.abs(K - Ko).max()
    print(f"{mode}: split K vs oracle {err:.2e}")
    assert err <= 1e-11
    assert np.array_equal(eng.hjk_computed(len(P["launches"])), _kept_per_launch(eng, P))


@pytest.mark.parametrize("tau", [1e-12, 1e-8])
def test_split_k_screen_matches_the_plan(cuda, lib_built, tau):
    """c0: the device skips exactly the visits the plan skips, and the
    screened K differs from the unscreened one by no more than the sum of
    the skipped visits' keys times the block sizes bound."""
    import torch
    w = configs.c0()
    eng = FockEngine(w.basis)
    D = torch.tensor(w.D, device=cuda)
    eng.hjk_plan(w.D, 0.0, mode="canonical", screen="k")
    K0 = eng.hjk_k(D).clone()
    P = eng.hjk_plan(w.D, tau, mode="canonical", screen="k")
    K1 = eng.hjk_k(D)
    kept = _kept_per_launch(eng, P)
    got = eng.hjk_computed(len(P["launches"]))
    assert np.array_equal(got, kept)
    assert int(got.sum()) == P["counts"]["quartets"] - P["counts"]["quartets_skipped"]
    d = float((K1 - K0).abs().max())
    bound = P["counts"]["quartets_skipped"] * tau * 36  # at most 6 x 6 elements of a d block a deposit
    print(f"tau {tau}: {P['counts']['quartets_skipped']} skipped, max|dK| {d:.2e} (bound {bound:.1e})")
    assert d <= bound


def test_split_k_matches_fused_build(cuda, lib_built):
    """c0 at its tau: the split stream's K against the fused build's K."""
    import torch
    w = configs.c0()
    eng = FockEngine(w.basis)
    eng.plan(w.D, 0.0, 4)
    D = torch.tensor(w.D, device=cuda)
    _, Kf, _ = eng.build(D)
    eng.hjk_plan(w.D, 0.0, mode="ordered", screen="k")
    K = eng.hjk_k(D)
    assert float((K - Kf).abs().max()) <= 1e-11


def test_refuses_a_j_keyed_stream(cuda, lib_built):
    import torch
    w = configs.cluster(1, 3)
    eng = FockEngine(w.basis)
    eng.hjk_plan(w.D, 1e-12, screen="j")
    with pytest.raises(Exception, match="J's key"):
        eng.hjk_k(torch.tensor(w.D, device=cuda))
