"""Algorithmic FLOPs of a computed quartet: the reference's own FLOP model.

`data/hgp_cost.json` holds, per class (la lb | lc ld) with every shell l <= 3,
the reference's `hgp.cost.cost(cls)` tiers (hgp/cost.py:199-245: one +, -,
*, / = one flop, no FMA fusion; Boys, exp and rsqrt named apart), written
by tests/golden/make_golden.py.  A quartet with contraction degrees K_AB,
K_CD costs

    x K_AB K_CD + y_bra K_AB + y_ket K_CD + z + 12 n_eri

the last term being the six-block digest (6 multiply-adds per ERI).
"""

from __future__ import annotations

import json
import os
from functools import lru_cache

HERE = os.path.dirname(os.path.abspath(__file__))


@lru_cache(maxsize=1)
def table() -> dict[tuple[int, int, int, int], dict]:
    with open(os.path.join(HERE, "data", "hgp_cost.json")) as f:
        d = json.load(f)
    return {tuple(r["class"]): r for r in d["classes"]}


def quartet_flops(cls, kab: int, kcd: int) -> int:
    r = table()[tuple(cls)]
    return (r["x"] * kab * kcd + r["y_bra"] * kab + r["y_ket"] * kcd + r["z"]
            + 12 * r["n_eri"])


def build_flops(launch_stats) -> dict[tuple[int, int, int, int], float]:
    """Per class, the algorithmic FLOPs of the quartets a build computed."""
    out: dict[tuple[int, int, int, int], float] = {}
    for s in launch_stats:
        cls = (s["la"], s["lb"], s["lc"], s["ld"])
        out[cls] = out.get(cls, 0.0) + float(s["computed"]) * quartet_flops(cls, s["kab"], s["kcd"])
    return out
