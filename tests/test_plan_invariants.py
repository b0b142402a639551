"""Invariants of the two host plans, on seeded workloads and thresholds where
pruning, deletion and the pre-launch screen all act (host-only handles).

F plan (eri/fock/launch_f.py; walk_f.py:320-330 refuses a plan otherwise):
the batch pairs I <= J are exactly the launches plus the pre-launch screened
ones, each once; every unique quartet of shell pairs is launched, screened
or lost to a deleted pair, exactly once; each batch is degree-uniform and
sorted descending by key.
J plan (eri/j_coulomb/launch.py:274-327): every record lies in one L group,
the ket order of each L is a permutation of that group, its keys do not
increase, and ties keep sweep order (stable)."""

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine


@pytest.mark.parametrize("wname,tau", [("c0", 1e-12), ("c0", 1e-6), ("cluster4", 1e-9), ("cluster6", 1e-4)])
def test_f_plan_partitions_the_quartets(lib_built, wname, tau):
    w = configs.by_name(wname)
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, tau, w.n_mag)
    nb = len(P.batches)
    launched = {(L.bra, L.ket) for L in P.launches}
    screened = set(map(tuple, P.screened))
    assert len(launched) == len(P.launches) and len(screened) == len(P.screened)
    assert not launched & screened
    assert launched | screened == {(i, j) for i in range(nb) for j in range(i, nb)}

    def quartets(i, j):
        ni, nj = len(P.batches[i].pairs), len(P.batches[j].pairs)
        return ni * (ni + 1) // 2 if i == j else ni * nj

    n_kept = sum(len(b.pairs) for b in P.batches)
    n_del = len(P.deleted)
    nsh = len(w.basis.shells)
    assert n_kept + n_del == nsh * (nsh + 1) // 2
    total = (n_kept + n_del) * (n_kept + n_del + 1) // 2
    lost = n_del * n_kept + n_del * (n_del + 1) // 2
    assert sum(quartets(*x) for x in launched) + sum(quartets(*x) for x in screened) + lost == total
    assert sum(quartets(*x) for x in launched) == P.quartets_launched
    for b in P.batches:
        assert len({p.degree for p in b.pairs}) == 1
        keys = [p.key for p in b.pairs]
        assert all(k0 >= k1 for k0, k1 in zip(keys, keys[1:]))


@pytest.mark.parametrize("wname", ["c0", "cluster5"])
def test_j_plan_ket_order(lib_built, wname):
    w = configs.by_name(wname)
    lst = FockEngine(w.basis, device=-1).j_plan_lists(w.D)
    L, key, order, off = lst["L"], lst["key"], lst["ket_order"], lst["L_off"]
    assert off[0] == 0 and off[-1] == len(L)
    for l in range(len(off) - 1):
        o = order[off[l]:off[l + 1]]
        assert np.array_equal(np.sort(o), np.flatnonzero(L == l))
        k = key[o]
        assert np.all(k[:-1] >= k[1:])
        ties = np.flatnonzero(k[:-1] == k[1:])
        assert np.all(o[ties] < o[ties + 1])  # stable
