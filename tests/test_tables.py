"""The shipped tables the build reads: the reference's FLOP model per class
(data/hgp_cost.json, the roofline's numerator) and the autotuner's
per-class launch choices (data/class_config.json)."""

import itertools

import pytest

from felizjueves_b200 import autotune, cost


def _classes():
    out = []
    for la, lb, lc, ld in itertools.product(range(4), repeat=4):
        if la <= lb and lc <= ld and (la, lb) <= (lc, ld):
            out.append((la, lb, lc, ld))
    return out


def test_cost_table_covers_every_class():
    t = cost.table()
    assert sorted(t) == sorted(_classes())  # 55 classes to (ff|ff)
    assert cost.quartet_flops((0, 0, 0, 0), 1, 1) == 18 + 20 + 20 + 16 + 12
    for cls in _classes():
        n = 1
        for l in cls:  # noqa: E741
            n *= (l + 1) * (l + 2) // 2
        assert t[cls]["n_eri"] == n
        # more primitives never cost less
        assert cost.quartet_flops(cls, 3, 2) > cost.quartet_flops(cls, 2, 2) > cost.quartet_flops(cls, 1, 2)


def test_build_flops_sums_computed_quartets():
    stats = [dict(la=0, lb=0, lc=0, ld=0, kab=1, kcd=1, launched=10, computed=4),
             dict(la=0, lb=0, lc=0, ld=0, kab=2, kcd=1, launched=5, computed=5),
             dict(la=1, lb=1, lc=1, ld=1, kab=1, kcd=1, launched=3, computed=0)]
    f = cost.build_flops(stats)
    assert f[(0, 0, 0, 0)] == 4 * cost.quartet_flops((0, 0, 0, 0), 1, 1) + 5 * cost.quartet_flops((0, 0, 0, 0), 2, 1)
    assert f[(1, 1, 1, 1)] == 0.0


def test_shipped_class_config_is_consistent():
    t = autotune.load_default()
    assert t is not None and {"choice", "ms", "choice32", "ms32", "workload"} <= set(t)
    keys = {tuple(int(x) for x in k.split(",")) for k in t["choice"]}
    assert keys <= set(_classes())
    for k, c in t["choice"].items():
        assert tuple(c) in autotune.CANDIDATES
        # the choice is the fastest candidate measured for the class
        ms = t["ms"][k]
        assert ms[f"{c[0]}x{c[1]}"] == pytest.approx(min(ms.values()))
    for k, c in t["choice32"].items():
        assert tuple(c) in autotune.CANDIDATES32
