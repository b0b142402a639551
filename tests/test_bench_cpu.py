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


def test_reference_arm_line_without_this_library(oracle_lib):
    """`bench.py --impl reference` on c0 prints one JSON line with the
    contract's keys, its cpu_baseline and zero-copy e2e describing the same
    run, and never maps libfjb.so into its process."""
    import json
    import subprocess
    import sys
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'c0', '--steps', '1', '--warmup', '0']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "finally:\n"
        "    maps = open('/proc/self/maps').read()\n"
        "    print('LIBFJB_MAPPED' if 'libfjb' in maps else 'LIBFJB_ABSENT')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=HERE, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "LIBFJB_ABSENT"
    rec = json.loads([ln for ln in lines if ln.startswith("{")][-1])
    assert rec["impl"] == "reference" and rec["higher_is_better"] is False
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "config"):
        assert k in rec, k
    assert rec["value"] > 0 and rec["unit"] == "ms/iter"
    cb = rec["cpu_baseline"]
    assert cb["value"] == rec["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e = rec["e2e"]
    assert e["value"] == rec["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
