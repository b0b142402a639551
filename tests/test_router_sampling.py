"""The router's training sampler (router.plan_samples), host only: every
sampled (launch, bra, ket) names the plan's own pairs, the canonical half on
diagonal launches, and launches are drawn in proportion to the quartets they
hold; the c3 training systems are seeded and within 8-64 atoms."""

import numpy as np

from felizjueves_b200 import configs, router
from felizjueves_b200.fock import FockEngine


def test_plan_samples_name_the_plans_pairs(lib_built):
    w = configs.cluster(6, 11)
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, w.tau, w.n_mag)
    s, q = router.plan_samples(eng, 4000, np.random.default_rng(1))
    sizes = np.array([len(P.batches[L.bra].pairs) * len(P.batches[L.ket].pairs) for L in P.launches])
    for (l, ib, ik), qq in zip(s, q):
        L = P.launches[l]
        pb, pk = P.batches[L.bra].pairs[ib], P.batches[L.ket].pairs[ik]
        assert (pb.a, pb.b, pk.a, pk.b) == tuple(qq)
        assert L.bra != L.ket or ik >= ib
    # launches drawn by size: the largest launch is drawn about as often as its share
    big = int(np.argmax(sizes))
    share = sizes[big] / sizes.sum()
    got = np.mean(s[:, 0] == big)
    assert abs(got - share) < 5 * np.sqrt(share * (1 - share) / len(s)) + 1e-3


def test_c3_clusters_are_seeded_and_in_range():
    a = [w.n_ao for w in router.c3_clusters(n=5)]
    b = [w.n_ao for w in router.c3_clusters(n=5)]
    assert a == b
    for w in router.c3_clusters(n=5):
        atoms = len({s.centre for s in w.basis.shells})
        assert 8 <= atoms <= 64
