"""Per-class launch configuration chosen by measurement.

The reference picks a kernel's batch count from measured medians
(performance/dispatch.py:1-45).  Here the choice is per angular-momentum
class: the CTA width of its HGP kernel (and, optionally, the chunk of
primitive quartets a CTA pass holds).  Every candidate is applied to every
class at once, one build is timed per candidate with CUDA events around each
class kernel (`FockEngine.class_stats`), the medians over `reps` builds are
compared class by class, and the winner is set.
"""

from __future__ import annotations

import json
import os

import numpy as np

# (threads, slots): (1, 0) the register kernel; slots 0 the layout's default
# chunk, 1 the single-slot path forced
CANDIDATES = ((1, 0), (32, 0), (64, 0), (128, 0), (256, 0), (512, 0), (32, 1), (64, 1), (128, 1), (256, 1),
              (512, 1))


def autotune(eng, D, candidates=CANDIDATES, reps: int = 1, precision: int = 0) -> dict:
    import torch
    classes = [(r["la"], r["lb"], r["lc"], r["ld"]) for r in eng.class_stats()] \
        if _has_build(eng) else None
    if classes is None:
        eng.build(D, precision=precision)
        torch.cuda.synchronize()
        classes = [(r["la"], r["lb"], r["lc"], r["ld"]) for r in eng.class_stats()]
    times: dict[tuple, dict[tuple, float]] = {c: {} for c in classes}
    for cand in candidates:
        ok = []
        for c in classes:
            try:
                eng.set_class_config(c, *cand)
                ok.append(c)
            except ValueError:
                pass
        samples: dict[tuple, list[float]] = {c: [] for c in ok}
        for _ in range(reps):
            eng.build(D, precision=precision)
            torch.cuda.synchronize()
            for r in eng.class_stats():
                c = (r["la"], r["lb"], r["lc"], r["ld"])
                if c in samples:
                    samples[c].append(r["ms"])
        for c, v in samples.items():
            if v:
                times[c][cand] = float(np.median(v))
    choice = {}
    for c, t in times.items():
        if not t:
            continue
        best = min(t, key=t.get)
        choice[c] = best
        eng.set_class_config(c, *best)
    return {"choice": {",".join(map(str, c)): list(v) for c, v in choice.items()},
            "ms": {",".join(map(str, c)): {f"{k[0]}x{k[1]}": v for k, v in t.items()}
                   for c, t in times.items()}}


CANDIDATES32 = ((32, 0), (64, 0), (128, 0), (256, 0), (512, 0), (32, 1), (64, 1), (128, 1), (256, 1), (512, 1),
                (128, 2))


def autotune32(eng, D, candidates=CANDIDATES32, reps: int = 1) -> dict:
    """The routed path's FP32 interpreter, per class: every unit sent to FP32
    (a routing threshold above every bound), one build timed per candidate
    (threads, slots), the fastest kept per class (classes with an FP32
    register body run it whatever this sets)."""
    import torch
    from . import _lib
    everything = 1e300
    times: dict[tuple, dict[tuple, float]] = {}
    for cand in candidates:
        classes = [(r["la"], r["lb"], r["lc"], r["ld"]) for r in eng.class_stats()] if times else None
        if classes is None:
            eng.build(D, precision=_lib.FJB_ROUTED, threshold=everything)
            torch.cuda.synchronize()
            classes = [(r["la"], r["lb"], r["lc"], r["ld"]) for r in eng.class_stats()]
            times = {c: {} for c in classes}
        ok = []
        for c in classes:
            try:
                eng.set_class_config32(c, *cand)
                ok.append(c)
            except ValueError:
                pass
        samples: dict[tuple, list[float]] = {c: [] for c in ok}
        for _ in range(reps):
            eng.build(D, precision=_lib.FJB_ROUTED, threshold=everything)
            torch.cuda.synchronize()
            for r in eng.class_stats():
                c = (r["la"], r["lb"], r["lc"], r["ld"])
                if c in samples:
                    samples[c].append(r["ms"])
        for c, v in samples.items():
            if v:
                times[c][cand] = float(np.median(v))
    choice = {}
    for c, t in times.items():
        if t:
            choice[c] = min(t, key=t.get)
            eng.set_class_config32(c, *choice[c])
    return {"choice32": {",".join(map(str, c)): list(v) for c, v in choice.items()},
            "ms32": {",".join(map(str, c)): {f"{k[0]}x{k[1]}": v for k, v in t.items()}
                     for c, t in times.items()}}


def _has_build(eng) -> bool:
    try:
        eng.class_stats()
        return True
    except Exception:
        return False


def apply(eng, table: dict) -> None:
    for key, (threads, slots) in table["choice"].items():
        try:
            eng.set_class_config(tuple(int(x) for x in key.split(",")), threads, slots)
        except ValueError:
            pass
    for key, (threads, slots) in table.get("choice32", {}).items():
        try:
            eng.set_class_config32(tuple(int(x) for x in key.split(",")), threads, slots)
        except ValueError:
            pass


def save(table: dict, path: str) -> None:
    with open(path, "w") as f:
        json.dump(table, f, indent=1)


DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                             "class_config.json")


def load_default() -> dict | None:
    """The shipped per-class choice (made by `autotune` on the 64-atom
    cluster on a B200), or None."""
    if not os.path.exists(DEFAULT_TABLE):
        return None
    with open(DEFAULT_TABLE) as f:
        return json.load(f)
