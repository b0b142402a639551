"""The bench's CPU baseline and reference arm, on the host: the shell-block
density maxima, the reference plan's loading, and the sampled estimate of a
whole build on the oracle (a small workload, a small budget)."""

import importlib.util
import os

import numpy as np

from felizjueves_b200 import configs

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_density_blocks_is_the_blockwise_max():
    b = _bench()
    w = configs.c0()
    Dsh = b.density_blocks(w.D, w.basis)
    off, sh = w.basis.offsets, w.basis.shells
    for s in range(0, len(sh), 7):
        for t in range(0, len(sh), 5):
            blk = w.D[off[s]:off[s] + sh[s].n_cart, off[t]:off[t] + sh[t].n_cart]
            assert Dsh[s, t] == np.abs(blk).max()


def test_cpu_estimate_on_the_reference_plan(oracle_lib):
    """c0: every launched quartet is sampled by key; the estimate is finite,
    positive, and scales with the thread count it divides by."""
    b = _bench()
    w = configs.c0()
    plan = b.reference_plan("c0")
    assert plan is not None and len(plan["launches"]) > 0
    ms, desc, spent = b.cpu_estimate(w, plan, w.D, cores=2, budget_s=0.5, seed=1)
    assert np.isfinite(ms) and ms > 0 and spent > 0
    assert "reference's own plan" in desc
