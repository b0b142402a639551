"""The split build's ordered pair stream built by libfjb (hjk_plan.cpp)
against the reference's own hjk_launches (eri/hjk/launch_hjk.py:280) on c0,
ordered mode, screens K and J at c0's tau and at 1e-6: pairs, batches,
launches and pair bounds bit-exact; every one of the 1.68 M visit keys
bit-exact (SHA-256 of them in visit order, and a strided sample), and the
skipped set the reference's (hash of the packed mask, and its first 2,000
indices).  Host-only handle (device -1): no GPU."""

import hashlib
import json

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine


@pytest.fixture(scope="module")
def c0():
    w = configs.c0()
    return w, FockEngine(w.basis, device=-1), golden("hjk_c0.npz")


def _visit_keys(eng, P):
    """Every visit's key and skip flag, in the plan's visit order."""
    keys, skipped = [], []
    b = P["batches"]
    for li, L in enumerate(P["launches"]):
        n = int(b[L[0], 4]) * int(b[L[1], 4])
        k, s = eng.hjk_keys(li, n)
        keys.append(k)
        skipped.append(s)
    return np.concatenate(keys), np.concatenate(skipped)


def test_pairs_batches_launches_bit_exact(lib_built, c0):
    w, eng, g = c0
    P = eng.hjk_plan(w.D, w.tau, mode="ordered", screen="k")
    assert np.array_equal(P["pairs"][:, :2], g["pair_ab"])
    assert np.array_equal(P["pairs"][:, 2:], g["pair_l_deg"])
    assert np.array_equal(P["batches"][:, :3], g["batch_key"])
    assert np.array_equal(P["batches"][:, 4], g["batch_npairs"])
    assert np.array_equal(P["launches"][:, :2], g["launches"])
    assert np.array_equal(P["launches"][:, 2:6], g["launch_cls"])
    # ordered mode: each launch on its own class, identity orientation
    assert np.array_equal(P["launches"][:, 6:10], g["launch_cls"])
    assert (P["launches"][:, 10:14] == [0, 1, 2, 3]).all()
    assert np.array_equal(P["pair_G"], g["pair_G"])


@pytest.mark.parametrize("screen", ["k", "j"])
@pytest.mark.parametrize("which", ["c0tau", "1e-6"])
def test_visit_keys_and_skips(lib_built, c0, screen, which):
    w, eng, g = c0
    tau = w.tau if which == "c0tau" else 1e-6
    P = eng.hjk_plan(w.D, tau, mode="ordered", screen=screen)
    tag = f"{screen}_{which}"
    assert P["counts"] == json.loads(str(g[f"{tag}_counts"]))
    keys, skipped = _visit_keys(eng, P)
    assert np.array_equal(keys[::997], g[f"{tag}_keys_sample"])
    assert hashlib.sha256(keys.tobytes()).hexdigest() == str(g[f"{tag}_keys_sha256"])
    assert hashlib.sha256(np.packbits(skipped).tobytes()).hexdigest() == str(g[f"{tag}_skipped_sha256"])
    head = g[f"{tag}_skipped_head"]
    assert np.array_equal(np.nonzero(skipped)[0][: len(head)], head)


def test_canonical_mode_orients_onto_compiled_classes(lib_built, c0):
    """Canonical mode: the same launches and visits; each launch's kernel
    class has la <= lb, lc <= ld, (la, lb) <= (lc, ld) and is the ordered
    class permuted by its shells map, a member of the ERI's 8-fold group."""
    w, eng, g = c0
    P = eng.hjk_plan(w.D, w.tau, mode="canonical", screen="k")
    group = {(0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2),
             (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0), (3, 2, 1, 0)}
    assert np.array_equal(P["launches"][:, :6], np.hstack([g["launches"], g["launch_cls"]]))
    for row in P["launches"]:
        o, k, sh = row[2:6], row[6:10], tuple(row[10:14])
        assert sh in group
        assert tuple(o[list(sh)]) == tuple(k)
        assert k[0] <= k[1] and k[2] <= k[3] and (k[0], k[1]) <= (k[2], k[3])


def test_refusals(lib_built, c0):
    w, eng, _ = c0
    D = w.D.copy()
    D[0, 1] += 1e-3
    with pytest.raises(ValueError, match="symmetric"):
        eng.hjk_plan(D, w.tau)
    with pytest.raises(ValueError):
        eng.hjk_plan(w.D, -1.0)
    with pytest.raises(ValueError, match="mode"):
        eng.hjk_plan(w.D, w.tau, mode="sorted")
    with pytest.raises(ValueError, match="screen"):
        eng.hjk_plan(w.D, w.tau, screen="x")
