"""The seeded workloads: sizes the measurements and the golden fixtures
depend on (c0: 36 shells, 90 AO; c1: 512 shells, 1984 AO) and the c4 batch's
uneven size draw (3-40 atoms, seed 4), each molecule with an exactly
symmetric density."""

import numpy as np

from felizjueves_b200 import configs


def test_c0_c1_sizes():
    w0, w1 = configs.c0(), configs.c1()
    assert (len(w0.basis.shells), w0.n_ao) == (36, 90)
    assert (len(w1.basis.shells), w1.n_ao) == (512, 1984)
    for w in (w0, w1):
        assert np.array_equal(w.D, w.D.T)


def test_c4_batch_draw():
    ws = configs.c4(12)
    sizes = [len(w.coords) for w in ws]
    assert all(3 <= n <= 40 for n in sizes)
    assert sizes == [len(w.coords) for w in configs.c4(12)]  # seeded
    assert len(set(sizes)) > 3  # uneven
    for w in ws:
        assert w.n_ao == 31 * len(w.coords)
        assert np.array_equal(w.D, w.D.T)
