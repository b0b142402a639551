"""The six-block screen restated on the CPU (oracle/screen.py) against the
reference's own walk_f prediction, recorded by tests/golden/make_golden.py:
every launched quartet of c0 (part_screen_c0) and 16,800 sampled launched
quartets of the 64-atom c1 (part_screen_c1), bit-exact, on this package's
host plan (itself bit-exact with the reference's f_launches).  The device's
mask is held to the same records by the GPU tests."""

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine
from oracle import screen


def _decisions(wname, fixture):
    w = getattr(configs, wname)()
    z = golden(fixture)
    P = FockEngine(w.basis, device=-1).plan(w.D, w.tau, w.n_mag)
    rows = z["rows"].astype(np.int64)
    sh, Gb, Gk = [], [], []
    for li, ib, ik, _ in rows:
        L = P.launches[li]
        br, kt = P.batches[L.bra].pairs[ib], P.batches[L.ket].pairs[ik]
        sh.append((br.a, br.b, kt.a, kt.b))
        Gb.append(br.G)
        Gk.append(kt.G)
    off = w.basis.offsets
    Dsh = screen.density_blocks(w.D, off, [s.n_cart for s in w.basis.shells])
    skip = screen.six_block_skip(Dsh, np.asarray(sh), np.asarray(Gb), np.asarray(Gk), w.tau)
    return skip, rows[:, 3].astype(bool), P


def test_c0_every_launched_quartet():
    skip, ref, P = _decisions("c0", "screen_c0.npz")
    assert len(ref) == P.quartets_launched
    assert np.array_equal(skip, ref), int((skip != ref).sum())
    assert 0 < ref.sum() < len(ref)  # both outcomes occur


def test_c1_sampled_launched_quartets():
    """Per (class, K_AB, K_CD) key the 12 draws whose bound lies nearest tau
    and 8 at random: the decisions that a wrong association or weight would
    flip first."""
    skip, ref, P = _decisions("c1", "screen_c1_sample.npz")
    assert P.quartets_launched == int(golden("screen_c1_sample.npz")["n_launched"])
    assert np.array_equal(skip, ref), int((skip != ref).sum())
    assert 0 < ref.sum() < len(ref)


def test_a_planted_weight_error_is_seen():
    """The exchange blocks weighed 1 instead of 1/2 (a plausible slip)
    changes decisions near tau on the c1 sample: the check can fail."""
    saved = screen.ABS_WEIGHTS
    try:
        screen.ABS_WEIGHTS = (2.0, 2.0, 1.0, 1.0, 1.0, 1.0)
        skip, ref, _ = _decisions("c1", "screen_c1_sample.npz")
    finally:
        screen.ABS_WEIGHTS = saved
    assert not np.array_equal(skip, ref)
