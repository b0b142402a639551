"""The plan's work units (fjb_plan_units).  Host-only handles fill the list
on the host; device handles write it on the GPU from one span a launch with
the same code (write_span_units).  CPU: the host list against a plain Python
restatement of the order the class kernels take: class by class in (la, lb,
lc, ld) order, each class's launches in plan order, each bra pair's kets
(from the bra pair itself on a diagonal launch) in chunks of 32.  GPU: the
device list bit-exact with the host one, at 8 atoms and at c1 (43 M units)."""

import hashlib

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

CHUNK = 32


def _expected_units(P) -> np.ndarray:
    by_class: dict[tuple, list[int]] = {}
    for li, L in enumerate(P.launches):
        b, k = P.batches[L.bra], P.batches[L.ket]
        by_class.setdefault((b.la, b.lb, k.la, k.lb), []).append(li)
    rows = []
    for key in sorted(by_class):
        for li in by_class[key]:
            L = P.launches[li]
            nb, nk = len(P.batches[L.bra].pairs), len(P.batches[L.ket].pairs)
            diag = L.bra == L.ket
            for ib in range(nb):
                for k0 in range(ib if diag else 0, nk, CHUNK):
                    rows.append((li, ib, k0, min(nk, k0 + CHUNK)))
    return np.array(rows, np.int32).reshape(-1, 4)


@pytest.mark.parametrize("n_atoms,seed", [(3, 5), (8, 11)])
def test_host_units_follow_the_class_order(lib_built, n_atoms, seed):
    w = configs.cluster(n_atoms, seed)
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, w.tau, w.n_mag)
    got = eng.plan_units()
    exp = _expected_units(P)
    assert any(L.bra == L.ket for L in P.launches) and any(L.bra != L.ket for L in P.launches)
    assert np.array_equal(got, exp)


def _expected_units_np(P) -> np.ndarray:
    """The same order, vectorised per launch (batches of ~1,000 pairs)."""
    keys = [(P.batches[L.bra].la, P.batches[L.bra].lb, P.batches[L.ket].la, P.batches[L.ket].lb)
            for L in P.launches]
    parts = []
    for li in sorted(range(len(P.launches)), key=lambda i: (keys[i], i)):
        L = P.launches[li]
        nb, nk = len(P.batches[L.bra].pairs), len(P.batches[L.ket].pairs)
        if L.bra == L.ket:
            ib, k0 = np.triu_indices(nb)
            keep = (k0 - ib) % CHUNK == 0  # chunk starts from the bra pair itself
            ib, k0 = ib[keep], k0[keep]
        else:
            ib, k0 = np.meshgrid(np.arange(nb), np.arange(0, nk, CHUNK), indexing="ij")
            ib, k0 = ib.ravel(), k0.ravel()
        parts.append(np.stack([np.full(len(ib), li), ib, k0, np.minimum(nk, k0 + CHUNK)], axis=1))
    return np.concatenate(parts).astype(np.int32) if parts else np.zeros((0, 4), np.int32)


def test_host_units_at_4_6_million(lib_built):
    """A 32-atom cluster (4.6 M units, batches of up to 956 pairs): the
    closed forms of the diagonal launches' unit offsets at size."""
    w = configs.cluster(32, 5)
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, w.tau, w.n_mag)
    got = eng.plan_units()
    assert len(got) > 4_000_000
    assert np.array_equal(got, _expected_units_np(P))


def test_everything_screened_gives_no_units(lib_built):
    w = configs.cluster(2, 5)
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, 1e6, w.n_mag)
    assert len(P.launches) == 0 and eng.plan_units().shape == (0, 4)


def test_unit_buffer_too_small_is_refused(lib_built):
    import ctypes as C
    w = configs.cluster(2, 5)
    eng = FockEngine(w.basis, device=-1)
    eng.plan(w.D, w.tau, w.n_mag, export=False)
    n = len(eng.plan_units())
    out = np.zeros((n, 4), np.int32)
    m = C.c_int64()
    assert eng._L.fjb_plan_units(eng._h, out.ctypes.data, n - 1, C.byref(m)) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cluster8", "c1"])
def test_device_units_equal_host_units(cuda, lib_built, which):
    import time
    w = configs.cluster(8, 11) if which == "cluster8" else configs.c1()
    host = FockEngine(w.basis, device=-1)
    host.plan(w.D, w.tau, w.n_mag, export=False)
    dev = FockEngine(w.basis)
    dev.plan(w.D, w.tau, w.n_mag, export=False)
    t = time.perf_counter()
    dev.plan(w.D, w.tau, w.n_mag, export=False)
    t_plan = time.perf_counter() - t
    a, b = host.plan_units(), dev.plan_units()
    print(f"{which}: {len(a)} units, a device plan {t_plan:.3f} s, "
          f"sha256 {hashlib.sha256(b.tobytes()).hexdigest()[:16]}")
    assert a.shape == b.shape and np.array_equal(a, b)
