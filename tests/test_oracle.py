"""The CPU oracle (oracle/oracle.c) pinned to the reference's own outputs
(tests/golden/, written by tests/golden/make_golden.py from the reference's
Python) and to the libcint/PySCF vj/vk fixtures the reference tracks."""

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs


def test_boys_matches_reference_quadrature(oracle_lib):
    z = golden("boys_ref.npz")
    F = np.array([[oracle_lib.boys(int(m), float(t)) for t in z["T"]] for m in z["M"]])
    rel = np.abs(F - z["F"]) / np.abs(z["F"])
    assert rel.max() < 1e-14


@pytest.mark.parametrize("wname", ["c0", "c1"])
def test_eri_blocks_match_reference(oracle_lib, wname):
    w = getattr(configs, wname)()
    z = golden(f"eri_{wname}.npz")
    ob = oracle_lib.OracleBasis.of(w.basis)
    off, val, sc = z["offsets"], z["values"], z["scale"]  # each npz read decompresses
    for i, q in enumerate(z["quartets"]):
        lo, hi = off[i], off[i + 1]
        got = oracle_lib.eri_block(ob, *map(int, q))
        err = np.abs(got - val[lo:hi])
        assert np.all(err <= 1e-14 * sc[lo:hi] + 1e-300), (q, err.max())


def test_eri_blocks_match_reference_c1_sample(oracle_lib):
    """c1: 40 quartets per class (10,240), each checked at the reference's
    largest-|value| element, its largest-scale element and six drawn at
    random, to 1e-14 of the element's own scale.  The blocks are computed on
    every host thread (the oracle's ctypes calls release the GIL; the first
    call, which fills its quadrature table, runs alone)."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    w = configs.c1()
    z = golden("eri_c1_sample.npz")
    ob = oracle_lib.OracleBasis.of(w.basis)
    Q, off, el = z["quartets"], z["offsets"], z["element"]
    val, sc = z["values"], z["scale"]  # read once: the npz is not thread-safe

    def ratio(i):
        lo, hi = off[i], off[i + 1]
        got = oracle_lib.eri_block(ob, *map(int, Q[i]))[el[lo:hi]]
        err = np.abs(got - val[lo:hi])
        return float((err / (1e-14 * sc[lo:hi] + 1e-300)).max())

    r = [ratio(0)]
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        r += list(ex.map(ratio, range(1, len(Q)), chunksize=64))
    r = np.asarray(r)
    bad = np.flatnonzero(r > 1.0)
    assert bad.size == 0, [(tuple(Q[i]), r[i]) for i in bad[:5]]
    print(f"worst err/tol = {r.max():.3f}")


LIBCINT = ["h2_sto3g", "h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "h10_chain_ccpvdz", "co_ccpvtz"]


@pytest.mark.parametrize("name", LIBCINT)
def test_jk_matches_libcint(oracle_lib, name):
    g = golden(f"libcint_{name}.npz")
    ob = oracle_lib.OracleBasis.from_npz(g)
    J, K = oracle_lib.jk(ob, g["D"])
    assert np.abs(J - g["vj"]).max() <= 1e-12 * np.abs(g["vj"]).max()
    assert np.abs(K - g["vk"]).max() <= 1e-12 * np.abs(g["vk"]).max()


@pytest.mark.parametrize("name,atoms,wfn", [("c0_1at", 1, "c0"), ("c0_2at", 2, "c0"),
                                            ("c1_1at", 1, "c1")])
def test_jk_matches_reference_host_path(oracle_lib, name, atoms, wfn):
    """J and K of the reference's coulomb_matrix / exchange_matrix
    (eri/j_coulomb/j.py:436, eri/k_exchange/k.py:482) on nested systems."""
    w = configs.sub_workload(getattr(configs, wfn)(), atoms)
    g = golden(f"jk_{name}.npz")
    assert np.array_equal(g["D"], w.D)
    ob = oracle_lib.OracleBasis.of(w.basis)
    for ordered in (False, True):
        J, K = oracle_lib.jk(ob, w.D, ordered=ordered)
        scale = max(np.abs(g["J"]).max(), np.abs(g["K"]).max())
        assert np.abs(J - g["J"]).max() <= 1e-14 * scale * 10
        assert np.abs(K - g["K"]).max() <= 1e-14 * scale * 10


def test_ordered_and_unique_sweeps_agree(oracle_lib):
    w = configs.cluster(2, 3)
    ob = oracle_lib.OracleBasis.of(w.basis)
    J1, K1 = oracle_lib.jk(ob, w.D)
    J2, K2 = oracle_lib.jk(ob, w.D, ordered=True)
    s = max(np.abs(J1).max(), np.abs(K1).max())
    assert np.abs(J1 - J2).max() <= 1e-13 * s
    assert np.abs(K1 - K2).max() <= 1e-13 * s


def test_wrong_weight_fails(oracle_lib):
    """A planted mistake (the Coulomb blocks at weight 1, the predecessor's
    bug the reference documents at kernel_f.py:98-101) misses by far more than
    the tolerance: the check can fail."""
    w = configs.cluster(1, 3)
    ob = oracle_lib.OracleBasis.of(w.basis)
    J, K = oracle_lib.jk(ob, w.D)
    J2, _ = oracle_lib.jk(ob, w.D, ordered=True)
    wrong = 0.5 * J  # what weight 1 on the Coulomb blocks would give
    assert np.abs(wrong - J2).max() > 1e3 * 1e-13 * np.abs(J2).max()


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


@pytest.mark.parametrize("name", ["h2o_ccpvtz_jkfit_metric", "h2o_sto3g_jkfit_3c",
                                  "prim_spd_f_auxi_metric", "prim_spd_f_auxi_3c"])
def test_df_integrals_match_libcint(oracle_lib, name):
    """(P|Q) and (mn|P) by the oracle's eri_block with every aux primitive
    paired with a unit s function, against libcint's (the fixtures the
    reference tracks for eri/density_fit)."""
    from oracle import df as odf
    z = golden(f"df_{name}.npz")
    ao, aux = _df_bases(z)
    got = odf.metric(aux) if str(z["kind"]) == "metric" else odf.eri3(ao, aux)
    ref = z["value"]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_fock_quartets_equals_unique_sweep(oracle_lib):
    """The timed per-quartet sample function (ERI block + six-block digest)
    over every unique quartet of c0, closed, equals the orbit sweep."""
    from felizjueves_b200 import configs
    w = configs.c0()
    ob = oracle_lib.OracleBasis.of(w.basis)
    n = len(w.basis.shells)
    pairs = [(a, b) for a in range(n) for b in range(a, n)]
    qs, dg = [], []
    for P in range(len(pairs)):
        for Q in range(P, len(pairs)):
            (a, b), (c, d) = pairs[P], pairs[Q]
            qs.append((a, b, c, d))
            dg.append((0.5 if a == b else 1.0) * (0.5 if c == d else 1.0) * (0.5 if P == Q else 1.0))
    J, K, sec = oracle_lib.fock_quartets(ob, w.D, qs, dg, threads=4)
    Jo, Ko = oracle_lib.jk(ob, w.D)
    assert np.abs(J + J.T - Jo).max() <= 1e-12
    assert np.abs(K + K.T - Ko).max() <= 1e-12
    assert sec.shape == (len(qs),) and np.all(sec > 0)


@pytest.mark.parametrize("name", ["h2_sto3g", "h2o_sto3g", "h2o_631g"])
def test_schwarz_diagonal_matches_libcint(oracle_lib, name):
    """(mn|mn) of every AO pair by the oracle's eri_block over each shell
    pair's (ab|ab) (the diagonal of eri/schwarz.py:86-102) against libcint's
    int2e diagonal the reference tracks."""
    g = golden(f"libcint_{name}_schwarz.npz")
    ob = oracle_lib.OracleBasis.from_npz(g)
    nc = [int(x) for x in ob.ncart]
    off = np.concatenate([[0], np.cumsum(nc)])
    M = np.zeros((off[-1], off[-1]))
    for a in range(len(nc)):
        for b in range(len(nc)):
            blk = oracle_lib.eri_block(ob, a, b, a, b).reshape(nc[a], nc[b], nc[a], nc[b])
            for i in range(nc[a]):
                for j in range(nc[b]):
                    M[off[a] + i, off[b] + j] = blk[i, j, i, j]
    ref = g["int2e_diag"]
    assert np.abs(M - ref).max() <= 1e-12 * np.abs(ref).max()


ERI_LIBCINT = ["h2o_631g_eri", "hf_ccpvtz_eri", "hf_ccpvtz_eri_l9", "hf_ccpvtz_eri_l10",
               "hf_ccpvtz_eri_l11", "hf_ccpvtz_eri_l12"]


@pytest.mark.parametrize("name", ERI_LIBCINT)
def test_eri_blocks_match_libcint(oracle_lib, name):
    """libcint's Cartesian (ij|kl) blocks the reference tracks, one shell
    quartet per class (all 55 classes to (ff|ff) over the hf_ccpvtz files,
    a general contraction with H off every axis), against the oracle's
    eri_block, at the reference's own bar: 1e-12 of each element's scale
    (test/test_ao_eri.py test_block_matches_libcint)."""
    g = golden(f"libcint_{name}.npz")
    ob = oracle_lib.OracleBasis.from_npz(g)
    off, val = g["offsets"], g["values"]
    classes = set()
    for i, q in enumerate(g["quartets"]):
        got, sc = oracle_lib.eri_block(ob, *map(int, q), want_scale=True)
        ref = val[off[i]:off[i + 1]]
        err = np.abs(got - ref)
        assert np.all(err <= 1e-12 * sc), (tuple(q), float(err.max()))
        ls = [int(g["l"][s]) for s in q]
        classes.add(tuple(sorted((tuple(sorted(ls[:2])), tuple(sorted(ls[2:]))))))
    # one quartet per class under the ERI's 8-fold symmetry
    assert len(classes) == len(g["quartets"]) or name == "h2o_631g_eri"
