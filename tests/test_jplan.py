"""The J-engine's plan (eri/j_coulomb/launch.py:274-327) against the
reference's own launches() on c0 (tests/golden/jplan_c0.npz): the records
and their order, I_pair per record, and the ket order per Hermite order L
(descending key, stable) equal; the bounds and keys to rounding.  Host-only
handle: no GPU."""

import numpy as np

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

from conftest import golden


def test_j_plan_lists_match_reference_c0(lib_built):
    g = golden("jplan_c0.npz")
    w = configs.c0()
    eng = FockEngine(w.basis, device=-1)
    lst = eng.j_plan_lists(w.D)
    abp = np.stack([lst["a"], lst["b"], lst["prim"]], axis=1)
    n_checked = 0
    for L in range(7):
        if f"bra{L}_ijp" not in g.files:
            assert not np.any(lst["L"] == L)
            continue
        sel = np.flatnonzero(lst["L"] == L)  # sweep order within L: the bra list
        np.testing.assert_array_equal(abp[sel], g[f"bra{L}_ijp"])
        np.testing.assert_allclose(lst["G"][sel], g[f"bra{L}_G"], rtol=4e-16, atol=0)
        o0, o1 = lst["L_off"][L], lst["L_off"][L + 1]
        order = lst["ket_order"][o0:o1]
        np.testing.assert_array_equal(abp[order], g[f"ket{L}_ijp"])  # the sorted ket list, bit-exact
        np.testing.assert_allclose(lst["key"][order], g[f"ket{L}_key"], rtol=1e-15, atol=0)
        n_checked += len(sel)
    assert n_checked == len(lst["a"]) == 4746


def test_j_plan_lists_match_reference_c1(lib_built):
    """The same on the 64-atom c1 (tests/golden/jplan_c1.npz): per Hermite
    order L the record count, the bra records in sweep order and the ket
    records in sorted order to the bit (sha256 of the int32 (i, j, prim)
    rows), and every 64th record's I_pair and key to rounding."""
    import hashlib
    g = golden("jplan_c1.npz")
    w = configs.c1()
    lst = FockEngine(w.basis, device=-1).j_plan_lists(w.D)
    abp = np.stack([lst["a"], lst["b"], lst["prim"]], axis=1).astype(np.int32)
    k = int(g["stride"])
    n_checked = 0
    for L in range(7):
        if f"bra{L}_n" not in g.files:
            assert not np.any(lst["L"] == L)
            continue
        sel = np.flatnonzero(lst["L"] == L)
        assert len(sel) == int(g[f"bra{L}_n"])
        assert hashlib.sha256(np.ascontiguousarray(abp[sel]).tobytes()).hexdigest() == str(g[f"bra{L}_sha"])
        np.testing.assert_allclose(lst["G"][sel][::k], g[f"bra{L}_G"], rtol=4e-16, atol=0)
        o0, o1 = lst["L_off"][L], lst["L_off"][L + 1]
        order = lst["ket_order"][o0:o1]
        assert hashlib.sha256(np.ascontiguousarray(abp[order]).tobytes()).hexdigest() == str(g[f"ket{L}_sha"])
        np.testing.assert_allclose(lst["key"][order][::k], g[f"ket{L}_key"], rtol=1e-15, atol=0)
        n_checked += len(sel)
    assert n_checked == len(lst["a"])
