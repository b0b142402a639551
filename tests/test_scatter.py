"""The atomics-free write-back's maps (eri/fock/kernel_f_scatter.py:203-260)
against the reference's own scatter_map on c0 (tests/golden/scatter_c0.npz:
each class's first launch and its first diagonal one, 27 launches): the
elements, the CSR offsets and every slot index equal.  Host-only handle."""

import numpy as np

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

from conftest import golden


def test_scatter_maps_bit_exact_c0(lib_built):
    g = golden("scatter_c0.npz")
    w = configs.c0()
    eng = FockEngine(w.basis, device=-1)
    eng.plan(w.D, w.tau, w.n_mag)
    n_slots = 0
    for li, n_el, n_slot, el0, ptr0, src0 in g["meta"]:
        m = eng.scatter_map(int(li))
        assert m["el"].shape == (n_el, 2) and len(m["src"]) == n_slot
        np.testing.assert_array_equal(m["el"].ravel(), g["el"][2 * el0:2 * (el0 + n_el)])
        np.testing.assert_array_equal(m["ptr"], g["ptr"][ptr0:ptr0 + n_el + 1])
        np.testing.assert_array_equal(m["src"], g["src"][src0:src0 + n_slot])
        assert np.array_equal(np.sort(m["src"]), np.arange(n_slot))  # every slot once
        n_slots += n_slot
    assert len(g["meta"]) == 27 and n_slots == len(g["src"])


def test_scatter_maps_bit_exact_c1_sample(lib_built):
    """c1 (the 64-atom cluster): per (class, diagonal) key the launch with
    the fewest slots, where the reference's pure-Python scatter_map is
    affordable (19 launches, 0.97 M slots; tests/golden/make_golden.py
    part_scatter_c1): counts and every map array to the bit (sha256)."""
    import hashlib
    g = golden("scatter_c1.npz")
    w = configs.c1()
    eng = FockEngine(w.basis, device=-1)
    eng.plan(w.D, w.tau, w.n_mag)
    for (li, n_el, n_slot), sha in zip(g["meta"], g["sha"]):
        m = eng.scatter_map(int(li))
        assert m["el"].shape == (n_el, 2) and len(m["src"]) == n_slot
        got = [hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()
               for a in (m["el"].ravel(), m["ptr"], m["src"])]
        assert got == [str(x) for x in sha], int(li)
