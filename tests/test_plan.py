"""The pair stream built by libfjb (plan.cpp) against the reference's own
f_launches (eri/fock/launch_f.py:390) on the seeded workloads: every integer
list and bound bit-exact.  Runs through the C ABI on a host-only
handle (device -1): no GPU."""

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine


def _plan(wname):
    w = getattr(configs, wname)()
    e = FockEngine(w.basis, device=-1)
    return w, e.plan(w.D, w.tau, w.n_mag)


@pytest.mark.parametrize("wname", ["c0", "c1"])
def test_plan_lists_bit_exact(lib_built, wname):
    w, P = _plan(wname)
    g = golden(f"plan_{wname}.npz")
    pairs = P.pairs
    assert np.array_equal(np.array([(b.la, b.lb, b.degree, b.mag) for b in P.batches]),
                          g["batch_key"])
    assert np.array_equal(np.array([len(b.pairs) for b in P.batches]), g["batch_npairs"])
    assert np.array_equal(np.array([(p.a, p.b) for p in pairs]), g["pair_ab"])
    assert np.array_equal(np.array([k for p in pairs for k in p.prims]), g["prims"])
    assert np.array_equal(np.array([p.mag for p in pairs]), g["pair_mag"])
    assert np.array_equal(np.array([(L.bra, L.ket) for L in P.launches]).reshape(-1, 2),
                          g["launches"])
    assert np.array_equal(np.array(P.screened).reshape(-1, 2), g["screened"])
    assert np.array_equal(np.array(P.deleted).reshape(-1, 2), g["deleted"])
    assert P.magnitudes == tuple(g["magnitudes"])
    assert P.eps == float(g["eps"]) and P.g_max == float(g["g_max"])
    assert P.n_prim_total == int(g["n_prim_total"])
    # bounds: to the bit (F_m(0) is the reference's own quadrature value)
    G = np.array([p.G for p in pairs])
    assert np.array_equal(G, g["pair_G"])
    assert np.array_equal(np.array([p.dmax for p in pairs]), g["pair_dmax"])
    import json
    assert P.counts() == json.loads(str(g["counts"]))


def test_c0_counts(lib_built):
    _, P = _plan("c0")
    assert P.counts() == {"pairs": 666, "pairs_deleted": 122, "primitive_pairs": 4746,
                          "primitive_pairs_pruned": 1784, "batches": 48,
                          "batch_pairs": 1176, "batch_pairs_screened": 306,
                          "launches": 870}


def test_batches_sorted_and_degree_uniform(lib_built):
    _, P = _plan("c0")
    keys = [(b.la, b.lb, b.degree, b.mag) for b in P.batches]
    assert keys == sorted(keys)
    for b in P.batches:
        assert all(p.degree == b.degree for p in b.pairs)
        k = [p.key for p in b.pairs]
        assert all(k[i] >= k[i + 1] for i in range(len(k) - 1))
    for L in P.launches:
        assert L.bra <= L.ket
        assert P.batches[L.bra].mag + P.batches[L.ket].mag < P.n


def test_prelaunch_screen_is_sound(lib_built):
    _, P = _plan("c0")
    for i, j in P.screened:
        assert P.batches[i].g_max * P.batches[j].g_max < P.tau


def test_tau_zero_deletes_nothing(lib_built):
    w = configs.c0()
    e = FockEngine(w.basis, device=-1)
    P = e.plan(w.D, 0.0, 4)
    assert P.deleted == () and P.screened == ()
    assert P.n_prim_kept == P.n_prim_total


def test_refusals(lib_built):
    w = configs.c0()
    e = FockEngine(w.basis, device=-1)
    D = w.D.copy()
    D[0, 1] += 1e-15
    with pytest.raises(ValueError, match="not symmetric"):
        e.plan(D, 1e-12, 4)
    D = w.D.copy()
    D[3, 3] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        e.plan(D, 1e-12, 4)
    with pytest.raises(ValueError, match="tau"):
        e.plan(w.D, -1.0, 4)
    with pytest.raises(ValueError, match="n ="):
        e.plan(w.D, 1e-12, 0)
    with pytest.raises(ValueError):
        e.plan(w.D[:5, :5], 1e-12, 4)
    with pytest.raises(RuntimeError, match="no plan|host-only"):
        FockEngine(w.basis, device=-1).build_host(w.D)


def test_l_above_limit_refused(lib_built):
    from felizjueves_b200.shell import Basis, Shell
    B = Basis((Shell(4, (0.0, 0.0, 0.0), [1.0], [1.0]),))
    with pytest.raises(ValueError, match="above the compiled maximum"):
        FockEngine(B, device=-1)


def test_pair_degree_limit(lib_built):
    """A shell pair of more than MAX_PRIM_PAIRS = 128 primitive pairs is
    refused (the interpreter stages a pair's primitives in shared memory,
    kernel_f.py:196-203); 11 x 11 = 121 is planned whole."""
    from felizjueves_b200.shell import Basis, Shell
    ex = list(np.geomspace(0.1, 50.0, 12))
    B = Basis((Shell(0, (0.0, 0.0, 0.0), ex, [1.0] * 12),))
    with pytest.raises(ValueError, match="MAX_PRIM_PAIRS"):
        FockEngine(B, device=-1).plan(np.ones((1, 1)), 0.0, 4)
    B = Basis((Shell(0, (0.0, 0.0, 0.0), ex[:11], [1.0] * 11),))
    P = FockEngine(B, device=-1).plan(np.ones((1, 1)), 0.0, 4)
    assert [b.degree for b in P.batches] == [121]


def test_one_electron_refusals(lib_built):
    """Nuclei are checked before any device work, as the reference's
    _check_nuclei (one_electron/potential.py:67-76) does."""
    w = configs.c0()
    e = FockEngine(w.basis, device=-1)
    with pytest.raises(ValueError, match="not \\(Z, centre\\)"):
        e.one_electron([(1.0,)])
    with pytest.raises(ValueError, match="three coordinates"):
        e.one_electron([(1.0, (0.0, 0.0))])
    with pytest.raises(ValueError, match="non-finite"):
        e.one_electron([(float("nan"), (0.0, 0.0, 0.0))])


def test_replan_reuses_bounds_with_identical_lists(lib_built):
    """A handle computes the D-independent pair bounds once and reuses them
    for later densities: each plan equals a fresh handle's plan."""
    w = configs.c0()
    e = FockEngine(w.basis, device=-1)
    for it in range(3):
        D = configs.perturbed_density(w.D, it)
        P = e.plan(D, w.tau, w.n_mag)
        Q = FockEngine(w.basis, device=-1).plan(D, w.tau, w.n_mag)
        assert P.launches == Q.launches and P.screened == Q.screened and P.deleted == Q.deleted
        assert [(b.la, b.lb, b.degree, b.mag) for b in P.batches] == [(b.la, b.lb, b.degree, b.mag) for b in Q.batches]
        assert [[(p.a, p.b, p.prims, p.G, p.key) for p in b.pairs] for b in P.batches] == \
               [[(p.a, p.b, p.prims, p.G, p.key) for p in b.pairs] for b in Q.batches]
