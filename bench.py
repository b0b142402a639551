"""Benchmark: the G = J - K/2 build of the 64-atom L<=3 cluster on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl fjb|reference]
                    [--precision fp64|routed]

One step = one fused J/K/G build of the 64-atom cluster (512 shells, s x3,
p x2, d x2, f x1 per atom, 1984 Cartesian AO, tau = 1e-12) for the step's
density D_k = D + 1e-3 sym(N(0,1)) (the SCF-like sequence, seeded per
iteration), every D_k resident in HBM before the timed region.  The plan is
built once (it depends on (basis, tau) and orders pairs by the first D);
each build screens with its own D_k.  The working set (D_k, J', K', J, K, G:
6 x 31.5 MB plus the staged pairs) exceeds the 126 MB L2, so no flush is
needed between steps.

Prints ONE JSON line (rank 0).  With N > 1 (torchrun), every rank builds its
own replica (the path is one molecule per GPU: "replicas only"), timed with
CUDA events, max over ranks.

--impl reference times the reference's CPU path, restated as the oracle
(oracle/oracle.c), on a bounded sample of the same workload's quartets with
every host core, and extrapolates to the whole build.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "G=J−K/2 build ms/iter: routed mixed vs plain FP64, same B200, |ΔG|≤1e-8"
WORKLOAD = ("64-atom cluster (seed 1, 0.1 atoms/A^3, >=0.95 A), per atom s x3 p x2 d x2 f x1 "
            "even-tempered Cartesian shells: 512 shells, 1984 AO; tau 1e-12, 4 eq.29 "
            "magnitudes; 20 SCF-like densities D_k = D + 1e-3 sym(N(0,1))")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fjb", choices=["fjb", "reference"])
    ap.add_argument("--precision", default="routed", choices=["fp64", "routed"])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--path", default="fock", choices=["fock", "coulomb", "df", "batch", "onee", "router"],
                    help="fock: the G build (the headline); coulomb: the MMD J-engine; "
                         "df: DF-J/K (FP64 and split-BF16 tensor-core GEMMs); batch: the "
                         "uneven molecule batch (c4) as one captured graph")
    ap.add_argument("--molecules", type=int, default=64, help="batch path: the first N c4 molecules")
    ap.add_argument("--atoms", type=int, default=16, help="df path: atoms of the c1-recipe cluster")
    ap.add_argument("--clusters", type=int, default=200, help="router path: c3 training clusters (8-64 atoms)")
    ap.add_argument("--router-samples", type=int, default=60000,
                    help="router path: launched quartets sampled per training cluster")
    ap.add_argument("--router-out", default="",
                    help="router path: where to save the trained network (.npz)")
    ap.add_argument("--router-label", default="deposit", choices=["deposit", "fp32_error"],
                    help="router path: train on each quartet's largest deposit (log10) or on its "
                         "largest FP32 error into G (the FP32 tap against the FP64 one)")
    ap.add_argument("--router-threshold", type=float, default=1e-9,
                    help="router path: the routed builds' threshold")
    ap.add_argument("--router-in", default="",
                    help="router path: evaluate this trained network (.npz) instead of training one "
                         "(its reach from a fresh c3 sample)")
    ap.add_argument("--df-block", type=int, default=768,
                    help="streamed df path: aux functions per block of (mn|P) (n_ao^2 x block doubles)")
    ap.add_argument("--df-stream", action="store_true",
                    help="df path: the streamed build (DFEngine.jk_streamed) below 32 atoms too")
    ap.add_argument("--threshold", type=float, default=1e-7,
                    help="routed builds: the Schwarz x density bound under which a unit runs FP32; "
                         "1e-7 is the largest the on-device 1e-8 budget check passes at c1 "
                         "(3e-7 measures 7.8e-9 but is estimated over budget and re-run in FP64)")
    ap.add_argument("--budget-threshold", type=float, default=1e-9,
                    help="a second routed measurement at this threshold (config c2's 1e-9 rule), "
                         "reported with its max|dG| against the 1e-8 budget (0: skip)")
    ap.add_argument("--router", default="bound", choices=["learned", "bound"],
                    help="routed builds: the learned router (trained and calibrated before the "
                         "timed region) or the Schwarz x density bound alone")
    return ap.parse_args()


# --- clocks -----------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --- CPU baseline: the oracle on a bounded sample ---------------------------

def reference_plan(workload: str):
    """The reference's own plan of the workload (its f_launches output,
    eri/fock/launch_f.py:390, recorded by tests/golden/make_golden.py from
    the reference itself): pairs with their bounds G and kept primitive
    pairs, batches and launches.  None for a workload with no record."""
    path = os.path.join(HERE, "tests", "golden", f"plan_{workload}.npz")
    if not os.path.exists(path):
        return None
    z = np.load(path)
    pb = z["pair_batch"]
    n_b = len(z["batch_npairs"])
    first = np.searchsorted(pb, np.arange(n_b))
    return {"ab": z["pair_ab"], "G": z["pair_G"], "prims": z["prims"], "prim_off": z["prim_off"],
            "batch_key": z["batch_key"], "batch_first": first, "batch_n": z["batch_npairs"],
            "launches": z["launches"], "tau": float(z["tau"])}


def density_blocks(D, basis):
    """max |D| over each shell block (kernel_f.py:608-617), n_sh x n_sh."""
    off = basis.offsets
    nc = [s.n_cart for s in basis.shells]
    n = len(nc)
    A = np.abs(D)
    rows = np.stack([A[off[i]:off[i] + nc[i]].max(axis=0) for i in range(n)])
    return np.stack([rows[:, off[j]:off[j] + nc[j]].max(axis=1) for j in range(n)], axis=1)


def cpu_estimate(w, plan, D, cores: int, budget_s: float = 6.0, seed: int = 0):
    """ms of one whole build on `cores` host cores by the oracle (the
    reference's per-quartet work: ERI block over the plan's kept primitive
    pairs + the six-block digest), estimated from a timed sample.

    Per (class, K_AB, K_CD) launch key: 256 launched quartets drawn (launch
    by its quartet count, then bra and ket uniformly) and put through the
    reference's six-block screen with the plan's G (walk_f.py:344-351) give
    the key's computed fraction; computed quartets drawn the same way are
    timed (a pilot of 2 per key, then as many more as fill about `budget_s`
    s of CPU).  Estimate = sum over keys of launched x computed fraction x
    mean time per computed quartet, / cores (the sample ran on `cores`
    threads at once).  Returns (ms, description, cpu_seconds_timed)."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    ab, G, bk = plan["ab"], plan["G"], plan["batch_key"]
    first, nb = plan["batch_first"], plan["batch_n"]
    tau = plan["tau"]
    Dsh = density_blocks(D, w.basis)
    LI = plan["launches"][:, 0].astype(np.int64)
    LJ = plan["launches"][:, 1].astype(np.int64)
    nI, nJ = nb[LI].astype(np.int64), nb[LJ].astype(np.int64)
    diag = LI == LJ
    nq = np.where(diag, nI * (nI + 1) // 2, nI * nJ)
    keys = {}
    for li in range(len(LI)):
        k = (int(bk[LI[li]][0]), int(bk[LI[li]][1]), int(bk[LJ[li]][0]), int(bk[LJ[li]][1]),
             int(bk[LI[li]][2]), int(bk[LJ[li]][2]))
        keys.setdefault(k, []).append(li)
    keys = {k: np.asarray(v, np.int64) for k, v in sorted(keys.items())}

    def draw(k, m):
        ls = keys[k]
        wts = nq[ls].astype(np.float64)
        li = ls[rng.choice(len(ls), size=m, p=wts / wts.sum())]
        ib = (rng.random(m) * nI[li]).astype(np.int64)
        lo = np.where(diag[li], ib, 0)
        ik = lo + (rng.random(m) * (nJ[li] - lo)).astype(np.int64)
        pi, pk = first[LI[li]] + ib, first[LJ[li]] + ik
        a, b, c, d = ab[pi, 0], ab[pi, 1], ab[pk, 0], ab[pk, 1]
        dmax = np.maximum.reduce([2.0 * Dsh[a, b], 2.0 * Dsh[c, d], 0.5 * Dsh[a, c],
                                  0.5 * Dsh[a, d], 0.5 * Dsh[b, c], 0.5 * Dsh[b, d]])
        on = ~(G[pi] * (G[pk] * dmax) < tau)
        same = diag[li] & (ib == ik)
        return pi, pk, same, on

    frac, cand = {}, {}
    for k in keys:
        pi, pk, same, on = draw(k, 256)
        frac[k] = float(on.mean())
        cand[k] = (pi[on], pk[on], same[on])
    ob = O.OracleBasis.of(w.basis)
    po, prims = plan["prim_off"], plan["prims"]

    def run(items):
        qs, dg, kept, owner = [], [], [], []
        for k, (pi, pk, same) in items:
            for x, y, z in zip(pi, pk, same):
                a, b = ab[x]
                c, d = ab[y]
                qs.append((a, b, c, d))
                dg.append((0.5 if a == b else 1.0) * (0.5 if c == d else 1.0) * (0.5 if z else 1.0))
                kept.append((prims[po[x]:po[x + 1]], prims[po[y]:po[y + 1]]))
                owner.append(k)
        if not qs:
            return {}, 0.0
        _, _, sec = O.fock_quartets(ob, D, qs, dg, kept, threads=cores)
        per = {}
        for k, t in zip(owner, sec):
            per.setdefault(k, []).append(float(t))
        return per, float(sec.sum())

    def computed(k, m):
        got = [[], [], []]
        while len(got[0]) < m:
            pi, pk, same, on = draw(k, max(64, int(2 * m / max(frac[k], 1e-3))))
            for g, x in zip(got, (pi[on], pk[on], same[on])):
                g.extend(x.tolist())
        return tuple(np.asarray(g[:m]) for g in got)

    live = [k for k in keys if frac[k] > 0.0]
    per, spent = run([(k, tuple(x[:2] for x in cand[k])) for k in live])
    n_more = int(min(100, max(0.0, budget_s / max(spent, 1e-9) - 1.0) * 2))
    if n_more:
        more, s2 = run([(k, computed(k, n_more)) for k in live])
        spent += s2
        for k, v in more.items():
            per.setdefault(k, []).extend(v)
    n_timed = sum(len(v) for v in per.values())
    total = 0.0
    for k in live:
        total += float(nq[keys[k]].sum()) * frac[k] * float(np.mean(per[k]))
    ms = 1e3 * total / cores
    desc = (f"oracle (the reference's eri_block over the plan's kept primitive pairs + the six-block "
            f"digest) on {n_timed} sampled computed quartets of the reference's own plan of the "
            f"workload ({len(keys)} (class, K_AB, K_CD) keys); computed fraction per key from 256 "
            f"draws through the reference's six-block screen; mean time per key x launched x "
            f"fraction, summed, / {cores} threads (the sample ran on {cores} threads); "
            f"{spent:.1f} s of CPU timed")
    return ms, desc, spent


# --- the GPU arm --------------------------------------------------------------

def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_arm(a, rank, world)
    if a.path != "fock":
        return side_path(a, local)

    import torch
    from felizjueves_b200 import _lib, configs, cost, replicas
    from felizjueves_b200.fock import FockEngine

    torch.cuda.set_device(local)
    dist = replicas.init(world, "nccl")
    w = configs.by_name(a.workload)
    eng = FockEngine(w.basis, device=local)
    P = eng.plan(w.D, w.tau, w.n_mag)
    n = w.n_ao
    n_d = 20
    Ds = [torch.tensor(configs.perturbed_density(w.D, i), device=f"cuda:{local}")
          for i in range(n_d)]
    Dw = torch.empty((n, n), dtype=torch.float64, device=f"cuda:{local}")
    J = torch.empty((n, n), dtype=torch.float64, device=f"cuda:{local}")
    K = torch.empty_like(J)
    G = torch.empty_like(J)
    stream = torch.cuda.current_stream()

    def timed(prec, thr=0.0):
        """W untimed builds, then K builds between two events on the build
        stream (each step: the in-place update of the working density, then
        the build replayed as its captured CUDA graph), bracketed by barrier + synchronize; nvidia-smi sampled over
        the timed region.  Returns ms/build (max over ranks), clocks, the
        kernel launches per build, the class and launch statistics of the
        last build and a copy of its G."""
        for i in range(a.warmup):
            Dw.copy_(Ds[i % n_d])  # the SCF loop's in-place density update
            eng.build(Dw, J=J, K=K, G=G, precision=prec, threshold=thr, graph=True)
        torch.cuda.synchronize()
        clocks = Clocks(local)
        clocks.start()
        replicas.barrier(dist)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(a.steps):
            Dw.copy_(Ds[i % n_d])  # the SCF loop's in-place density update
            eng.build(Dw, J=J, K=K, G=G, precision=prec, threshold=thr, graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        replicas.barrier(dist)
        ck_ = clocks.stop()
        ms_ = replicas.max_over_ranks(dist, e0.elapsed_time(e1) / a.steps, f"cuda:{local}")
        return ms_, ck_, eng.last_build_stats()[1], eng.class_stats(), eng.launch_stats(), G.clone()

    ms64, ck64, nl64, cs, ls, G64 = timed(_lib.FJB_FP64)
    router_info = None
    if a.precision == "routed" and a.router == "learned":
        router_info = install_learned_router(eng, a.threshold)
    budget = None
    if a.precision == "routed":
        ms, ck, nl, cs_r, ls_r, Gr = timed(_lib.FJB_ROUTED, a.threshold)
        n32, n64 = route_counts(eng)
        est, rerouted = eng.route_check()
        router_info = dict(router_info or {"kind": "bound"}, fp32_units=n32, fp64_units=n64,
                           budget_check={"budget": 1e-8, "sample_stride": 32, "estimate": est,
                                         "rerouted_to_fp64": rerouted})
        if a.budget_threshold > 0:
            if a.router == "learned":
                install_learned_router(eng, a.budget_threshold)
            msb, _, _, _, _, Gb = timed(_lib.FJB_ROUTED, a.budget_threshold)
            estb, rrb = eng.route_check()
            budget = {"threshold": a.budget_threshold, "ms_per_step": round(msb, 3),
                      "speedup_vs_fp64": round(ms64 / msb, 4),
                      "max_abs_dG_vs_fp64": float((Gb - G64).abs().max()),
                      "fp32_units": route_counts(eng)[0],
                      "budget_check": {"estimate": estb, "rerouted_to_fp64": rrb}}
        dG = float((Gr - G64).abs().max())
        prec = _lib.FJB_ROUTED
    else:
        ms, ck, nl, cs_r, ls_r, dG = ms64, ck64, nl64, cs, ls, 0.0
        prec = _lib.FJB_FP64
    gpu_launches = nl * a.steps

    # roofline of the dominant class kernel of the plain FP64 build
    flops = cost.build_flops(ls)
    top = max(cs, key=lambda r: r["ms"])
    tcls = (top["la"], top["lb"], top["lc"], top["ld"])
    peak64 = ctypes_probe(_lib, 0)
    ach = flops.get(tcls, 0.0) / (top["ms"] * 1e-3) / 1e12
    build_tf = sum(flops.values()) / (sum(r["ms"] for r in cs) * 1e-3) / 1e12
    computed = sum(s["computed"] for s in ls)
    launched = sum(s["launched"] for s in ls)

    e2e = None
    if not a.no_e2e:
        # the same W + K sequence through the host-buffer C ABI: each step
        # copies its density in from pinned host memory and J, K, G out
        def pinned():
            return torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy()
        Dh = []
        for i in range(n_d):
            x = pinned()
            x[...] = configs.perturbed_density(w.D, i)
            Dh.append(x)
        outs = (pinned(), pinned(), pinned())
        for i in range(a.warmup):
            eng.build_host(Dh[i % n_d], precision=prec, threshold=a.threshold, out=outs)
        replicas.barrier(dist)
        t0 = time.perf_counter()
        for i in range(a.steps):
            eng.build_host(Dh[i % n_d], precision=prec, threshold=a.threshold, out=outs)
        e2e_ms = replicas.max_over_ranks(dist, (time.perf_counter() - t0) * 1e3 / a.steps,
                                         f"cuda:{local}")
        e2e = {"value": round(e2e_ms, 3), "unit": "ms/iter", "h2d_bytes_per_step": n * n * 8,
               "d2h_bytes_per_step": 3 * n * n * 8, "steps": a.steps, "warmup": a.warmup,
               "api": "fjb_fock_build_host (C ABI; pinned host buffers; H2D of D, build, D2H of "
                      "J, K, G inside the timed region, host clock, max over ranks)"}

    cpu = None
    if not a.no_cpu and rank == 0 and world == 1:
        plan = reference_plan(a.workload)
        if plan is not None:
            cores = os.cpu_count() or 1
            est, desc, spent = cpu_estimate(w, plan, configs.perturbed_density(w.D, 0), cores)
            cpu = {"value": round(est, 1), "unit": "ms/iter", "cores": cores, "kind": "port",
                   "estimate": "extrapolated from a timed sample", "sample": desc}

    out = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms/iter", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if a.precision == "fp64" else "f64+f32",
        "data": "synthetic (seeded cluster, random symmetric densities)",
        "precision": a.precision,
        "fp64": {"ms_per_step": round(ms64, 3), "clocks": ck64},
        "speedup_routed_vs_fp64": round(ms64 / ms, 4) if a.precision == "routed" else None,
        "max_abs_dG_vs_fp64": dG if a.precision == "routed" else None,
        "route_threshold": a.threshold if a.precision == "routed" else None,
        "routed_at_second_threshold": budget,
        "router": router_info,
        "config": {"workload": WORKLOAD, "n_ao": n, "shells": len(w.basis.shells),
                   "tau": w.tau, "quartets_launched": launched, "quartets_computed": computed,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "working set > 126 MB L2 (6 x 31.5 MB matrices + pair records); no flush"},
        "roofline": {"bound": "fp64",
                     "kernel": "%s class (%d%d|%d%d)" % (("hgp_fock_kernel", "hgp_compiled_kernel",
                                                          "rys_fock_kernel")[top.get("engine", 0)], *tcls),
                     "achieved": round(ach, 3), "peak": round(peak64, 3), "unit": "TFLOP/s",
                     "frac": round(ach / peak64, 4) if peak64 else None, "traffic": None,
                     "traffic_note": "not captured at this size; the kernel is FP64-issue and "
                                     "latency bound, its pair records and D read from L2: ncu "
                                     "measured 1.6 MB read + 23 MB written per launch of the "
                                     "(pp|pf) Rys class on a 16-atom cluster "
                                     "(profiles/rys_fock_kernel_pppf_cluster16.md)",
                     "peak_source": "measured: fjb_fma_probe FP64 FMA chains on this GPU "
                                    "(MEASURED_PEAKS.json has no FP64 figure)",
                     "build_tflops": round(build_tf, 3), "kernel_ms": round(top["ms"], 3),
                     "flop_model": "reference hgp/cost.py x K^4 + y K^2 + z + 12 n_eri"},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches, "clocks": ck,
    }
    if rank == 0:
        print(json.dumps(out))
    replicas.finish(dist)


def ctypes_probe(_lib, fp32: int) -> float:
    import ctypes as C
    v = C.c_double()
    _lib.check(_lib.load().fjb_fma_probe(fp32, 5, C.byref(v)))
    return float(v.value)


def install_learned_router(eng, threshold: float = 1e-9) -> dict:
    """The network trained for config c3 (router.load_default: 7.87 M FP64
    quartets of 200 seeded 8-64-atom clusters; bench.py --path router
    retrains it), installed on `eng` at the routed build's threshold with
    its calibrated margin, reach and class gate."""
    from felizjueves_b200 import router
    mlp, margin, reach, min_l = router.load_default(device=eng.device)
    router.install(eng, mlp, threshold=threshold, margin=margin, reach=reach, min_total_l=min_l)
    return {"kind": "learned", "training_quartets": 7867810, "margin_log10": round(margin, 3),
            "reach_decades": reach, "min_total_l": min_l}


def route_counts(eng):
    from felizjueves_b200 import router
    return router.route_stats(eng)


def side_path(a, local):
    """One GPU: the J-engine (`--path coulomb`: fjb_coulomb at the workload's
    tau) or DF-J/K (`--path df`: the (mn|P) L^-T factors once, then J and K
    per step in FP64 and as split-BF16 tensor-core GEMMs), W untimed and K
    timed steps with CUDA events on the current stream."""
    import torch
    from felizjueves_b200 import configs
    w = configs.by_name(a.workload)
    torch.cuda.set_device(local)
    D = torch.tensor(w.D, device=f"cuda:{local}")
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            out = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps, out

    line = {"n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "higher_is_better": False,
            "data": "synthetic", "dtype": "f64", "config": {"workload": a.workload, "n_ao": w.n_ao}}
    if a.path == "batch":
        return batch_path(a, local)
    if a.path == "router":
        return router_path(a, local)
    if a.path == "coulomb":
        from felizjueves_b200.fock import FockEngine
        eng = FockEngine(w.basis, device=local)
        J = torch.empty_like(D)
        ms, _ = timed(lambda: eng.coulomb(D, tau=w.tau, J=J))
        J64 = J.clone()
        ms32, _ = timed(lambda: eng.coulomb(D, tau=w.tau, J=J, threshold=a.threshold))
        line.update(metric="J-engine J build ms/iter", value=round(ms, 3), unit="ms/iter",
                    gpu_launches=eng.j_launches(),
                    fp32_tier={"threshold": a.threshold, "ms": round(ms32, 3),
                               "speedup_vs_fp64": round(ms / ms32, 4),
                               "max_abs_dJ_vs_fp64": float((J - J64).abs().max())})
    elif a.path == "onee":
        # S, T, V and H = T + V; one nucleus of charge 1 + (k mod 9) per atom
        from felizjueves_b200.fock import FockEngine
        centres = []
        for s_ in w.basis.shells:
            if s_.centre not in centres:
                centres.append(s_.centre)
        nuclei = [(float(1 + k % 9), c) for k, c in enumerate(centres)]
        eng = FockEngine(w.basis, device=local)
        outs = eng.one_electron(nuclei)
        ms, _ = timed(lambda: eng.one_electron(nuclei, S=outs[0], T=outs[1], V=outs[2], H=outs[3]))
        line.update(metric="one-electron S, T, V, H ms/iter", value=round(ms, 3), unit="ms/iter",
                    n_nuclei=len(nuclei), shell_pairs=len(w.basis.shells) * (len(w.basis.shells) + 1) // 2,
                    gpu_launches=10)
        if not a.no_cpu:
            # the oracle on a bounded sample of shell pairs, scaled by the pair count
            import random
            import time as _t
            from oracle import one_electron as _o
            rng = random.Random(0)
            sh = w.basis.shells
            pairs = [(i, j) for i in range(len(sh)) for j in range(i, len(sh))]
            sample = rng.sample(pairs, min(300, len(pairs)))
            t0 = _t.perf_counter()
            for i, j in sample:
                _o.blocks(sh[i], sh[j], nuclei)
            spent = _t.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(spent / len(sample) * len(pairs) * 1e3, 1), "unit": "ms/iter",
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle one_electron.blocks on {len(sample)} random shell pairs "
                                              f"of {len(pairs)}, {spent:.1f} s, scaled by the pair count"}
    elif a.atoms >= 32 or a.df_stream:
        return df_stream_path(a, local, line)
    else:
        # DF-J/K on a cluster of the c1 recipe (--atoms; the 64-atom system's
        # dense factors, 5,760 x 1,984^2 doubles, do not fit in HBM: from 32
        # atoms the streamed build, df_stream_path)
        from felizjueves_b200.df import DFEngine
        w = configs.cluster(a.atoms, 1)
        D = torch.tensor(w.D, device=f"cuda:{local}")
        aux = configs.aux_basis(w)
        eng = DFEngine(w.basis, aux, device=local)
        B = eng.factors()
        ms64, (J64, K64) = timed(lambda: eng.jk(D, "fp64", B=B))
        ms16, (J16, K16) = timed(lambda: eng.jk(D, "bf16x3", B=B))
        nq, n = aux.n_ao, w.n_ao
        useful = 4.0 * nq * n ** 3  # X = B D and K = sum_q X_q B_q^T, 2 nq n^3 flops each
        line.update(metric="DF-J/K ms/iter", value=round(ms16, 3), unit="ms/iter", dtype="bf16x3 -> f32",
                    config={"workload": f"{a.atoms}-atom cluster (c1 recipe), {n} AO, {nq} aux", "n_ao": n,
                            "n_aux": nq},
                    fp64_ms=round(ms64, 3), n_aux=nq,
                    k_gemm_useful_tflops=round(useful / (ms16 * 1e-3) / 1e12, 3),
                    k_gemm_tensor_tflops=round(6 * useful / (ms16 * 1e-3) / 1e12, 3),
                    gpu_launches=10,
                    max_abs_dJ_bf16x3_vs_fp64=float((J16 - J64).abs().max()),
                    max_abs_dK_bf16x3_vs_fp64=float((K16 - K64).abs().max()),
                    max_abs_K_fp64=float(K64.abs().max()))
    print(json.dumps(line))


def router_path(a, local):
    """Config c3: the learned router trained at scale -- `--clusters` seeded
    clusters of 8-64 atoms with the c1 shells, `--router-samples` launched
    quartets sampled from each, those the six-block screen computes labelled
    by the FP64 HGP tap (log10 of the largest deposit into G; with
    `--router-label fp32_error`, of the largest FP32 error into G), about 1e7
    in all -- on the GPU with the library's MLP kernels, calibrated on
    held-out quartets through the routing pass's tensor-core inference; then
    on the c1 system (not in the training set) the routed build at
    `--router-threshold` (1e-9) with the learned router (every class with
    its measured reach, every class with a 0.5-decade reach, and the shipped
    gate; or, for the error labels, three predicted-error thresholds)
    against the bound alone, all with the on-device budget check, against
    the FP64 build.  `--router-in` evaluates a trained network instead,
    its margin recalibrated on a fresh sample.  W warm-up and K timed graph
    replays each."""
    import time as _t
    import torch
    from felizjueves_b200 import _lib, configs, router
    from felizjueves_b200.fock import FockEngine
    torch.cuda.set_device(local)
    t0 = _t.perf_counter()
    if a.router_in:  # a trained network: a fresh sample of c3 systems for its reach and check
        z = np.load(a.router_in)
        X, y = router.training_set(router.c3_clusters(a.clusters, seed=7, first=20_000), n_per=a.router_samples,
                                   seed=5)
        va = np.arange(len(X))
        tr = np.arange(int(z["n_train"]))
        mlp = router.MLP(z["params"], device=local)
        # the margin recalibrated on the fresh, held-out sample, through the
        # routing pass's own arithmetic
        margin, losses, t_train = router.calibrate(mlp, X, y, 0.999), [float("nan")], 0.0
    else:
        X, y = router.training_set(router.c3_clusters(a.clusters), n_per=a.router_samples, seed=1,
                                   label=a.router_label)
        perm = np.random.default_rng(2).permutation(len(X))
        ntr = int(0.9 * len(X))
        tr, va = perm[:ntr], perm[ntr:]
        mlp = router.MLP(router.init_params(X[tr], y[tr], seed=0), device=local)
        t1 = _t.perf_counter()
        losses = mlp.train(X[tr], y[tr], epochs=12, batch=8192)
        torch.cuda.synchronize()
        t_train = _t.perf_counter() - t1
        margin = router.calibrate(mlp, X[va], y[va], 0.999)
    t_data = _t.perf_counter() - t0 - t_train
    rmse_va = float(np.sqrt(np.mean((y[va] - mlp.predict(X[va]).cpu().numpy()) ** 2)))
    reach = router.reach(mlp, X[va], margin)
    if a.router_out:
        gate = {"min_total_l": int(z["min_total_l"])} if a.router_in and "min_total_l" in z else {}
        np.savez(a.router_out, params=mlp.params(), margin=margin, reach=reach, n_train=len(tr), **gate)
    w = configs.c1()
    eng = FockEngine(w.basis, device=local)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=f"cuda:{local}")
    J, K, G = (torch.empty_like(D) for _ in range(3))
    st = torch.cuda.current_stream()

    def timed(prec, thr):
        for _ in range(max(1, a.warmup)):
            eng.build(D, J=J, K=K, G=G, precision=prec, threshold=thr, graph=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            eng.build(D, J=J, K=K, G=G, precision=prec, threshold=thr, graph=True)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps

    ms64 = timed(_lib.FJB_FP64, 0.0)
    G64 = G.clone()
    thr = a.router_threshold
    res = {}
    kinds = ("bound", "learned", "learned_r05", "learned_gated")
    if a.router_label == "fp32_error":  # the network routes by its predicted FP32 error
        kinds = ("bound", "err_1e-15", "err_1e-14", "err_1e-13")
    for kind in kinds:
        if kind.startswith("err_"):  # a unit's quartets each under the bound or predicted under this error
            router.install(eng, mlp, threshold=float(kind[4:]), margin=margin, reach=1.0)
        if kind == "learned":
            router.install(eng, mlp, threshold=thr, margin=margin, reach=reach)
        if kind == "learned_r05":  # every class, reach 0.5 decades
            router.install(eng, mlp, threshold=thr, margin=margin, reach=0.5)
        if kind == "learned_gated":  # the reach and class gate measured best on c1
            router.install(eng, mlp, threshold=thr, margin=margin, reach=0.5, min_total_l=7)
        ms = timed(_lib.FJB_ROUTED, thr)
        n32, n64 = router.route_stats(eng)
        est, rr = eng.route_check()
        res[kind] = {"ms_per_step": round(ms, 3), "speedup_vs_fp64": round(ms64 / ms, 4),
                     "max_abs_dG_vs_fp64": float((G - G64).abs().max()), "fp32_units": n32,
                     "fp64_units": n64, "budget_check": {"estimate": est, "rerouted_to_fp64": rr}}
    line = {"metric": f"learned router on c1: routed G build ms/iter at {thr:g} vs the bound alone",
            "value": res[kinds[1]]["ms_per_step"], "unit": "ms/iter", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "higher_is_better": False, "data": "synthetic", "dtype": "f64+f32",
            "config": {"workload": "c3: train on seeded 8-64-atom clusters, evaluate on c1",
                       "clusters": a.clusters, "samples_per_cluster": a.router_samples},
            "training_quartets": int(len(tr)), "validation_quartets": int(len(va)),
            "data_s": round(t_data, 1), "train_s": round(t_train, 1), "epochs": len(losses),
            "final_train_mse_log10": round(losses[-1], 5), "validation_rmse_log10": round(rmse_va, 4),
            "margin_log10": round(margin, 4), "reach_decades": reach, "fp64_ms_per_step": round(ms64, 3),
            "label": a.router_label, **res,
            **{f"{k}_gain_vs_bound": round(res["bound"]["ms_per_step"] / res[k]["ms_per_step"], 4)
               for k in kinds if k != "bound"}}
    print(json.dumps(line))


def df_stream_path(a, local, line):
    """Config c2's DF half at full size (`--path df --atoms 64`): the c1
    system with the even-tempered s..g aux basis (5,760 functions), DF-J/K
    by DFEngine.jk_streamed -- (mn|P) one aux block at a time from the
    three-centre Rys kernel, never held whole -- with K on the tensor cores
    (split BF16) and, once, in FP64; errors of both against the exact FP64
    build of the same density (the 4-centre fused build), per phase CUDA-event
    times.  The metric and its factor are set up once, outside the timed
    steps (as the dense path's factors are)."""
    import time as _t
    import torch
    from felizjueves_b200 import configs
    from felizjueves_b200.df import DFEngine
    from felizjueves_b200.fock import FockEngine
    w = configs.cluster(a.atoms, 1)
    dev = f"cuda:{local}"
    D = torch.tensor(w.D, device=dev)
    ex = FockEngine(w.basis, device=local)
    ex.plan(w.D, w.tau, w.n_mag)
    Jx, Kx, Gx = (t.clone() for t in ex.build(D))
    torch.cuda.synchronize()
    ex.close()
    del ex
    aux = configs.aux_basis(w)
    eng = DFEngine(w.basis, aux, device=local)
    t0 = _t.perf_counter()
    factor = eng.metric_factor()
    torch.cuda.synchronize()
    setup_s = _t.perf_counter() - t0
    st = torch.cuda.current_stream()

    def run(mode, n):
        tm = {}
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n):
            J, K = eng.jk_streamed(D, mode=mode, tau=w.tau, factor=factor, timings=tm, block=a.df_block)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, J, K, tm

    for _ in range(a.warmup):
        run("bf16x3", 1)
    ms, J, K, tm = run("bf16x3", a.steps)
    ms64, J64, K64, tm64 = run("fp64", 1)

    def err(X, R):
        return {"max_abs": float((X - R).abs().max()), "rel_max": float((X - R).abs().max() / R.abs().max())}

    G, G64 = J - 0.5 * K, J64 - 0.5 * K64
    nq, n = aux.n_ao, w.n_ao
    line.update(metric="DF-J/K ms/iter (streamed)", value=round(ms, 3), unit="ms/iter", dtype="f64; K bf16x3 -> f32",
                config={"workload": f"c2: {a.atoms}-atom c1-recipe cluster, {n} AO, {nq} aux (s..g, 0.1 2.2^k)",
                        "n_ao": n, "n_aux": nq, "aux_block_functions": a.df_block, "tau": w.tau},
                phases_ms={k: round(v, 3) if isinstance(v, float) else v for k, v in tm.items()},
                fp64_k_ms=round(ms64, 3), fp64_k_phases_ms={k: round(v, 3) if isinstance(v, float) else v
                                                            for k, v in tm64.items()},
                metric_setup_s=round(setup_s, 2),
                dJ_vs_exact=err(J, Jx), dK_vs_exact=err(K, Kx), dG_vs_exact=err(G, Gx),
                dK_bf16x3_vs_fp64_df=err(K, K64), dG_fp64_df_vs_exact=err(G64, Gx),
                gpu_launches=tm.get("fjb_launches"))
    print(json.dumps(line))


def batch_path(a, local):
    """The c4 batch (its first --molecules molecules): the plain FP64
    per-molecule loop (each molecule its own launches, one after another),
    then the batched build -- one launch per angular-momentum class for the
    whole batch over a class-sorted queue of every molecule's work units,
    captured as one CUDA graph -- in FP64 and routed (the Schwarz x density
    bound router at 1e-9); total ms per batch, per-molecule device ms of the
    loop (p50, p99) and max|dG| of the batched routed build against the
    per-molecule FP64 builds."""
    import torch
    from felizjueves_b200 import _lib, configs
    from felizjueves_b200.batch import BatchBuilder
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    ws = configs.c4(a.molecules)
    bb = BatchBuilder(ws, device=local)
    plan_s = time.perf_counter() - t0
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps

    loop_ms = timed(lambda: bb.build_loop(_lib.FJB_FP64))
    per = bb.device_ms()
    G64 = [g.clone() for g in bb.G()]
    bb.capture_merged("m64", _lib.FJB_FP64)
    m64_ms = timed(lambda: bb.replay("m64"))
    dG64 = max(float((g - h).abs().max()) for g, h in zip(bb.G(), G64))
    bb.capture_merged("m32", _lib.FJB_ROUTED, 1e-9)
    m32_ms = timed(lambda: bb.replay("m32"))
    dG = max(float((g - h).abs().max()) for g, h in zip(bb.G(), G64))
    # the learned router (config c3's trained network, installed on the
    # batch's first molecule: it routes them all)
    info = install_learned_router(bb.engines[0])
    n_tr = info["training_quartets"]
    bb.capture_merged("mlp", _lib.FJB_ROUTED, 1e-9)
    mlp_ms = timed(lambda: bb.replay("mlp"))
    dG_mlp = max(float((g - h).abs().max()) for g, h in zip(bb.G(), G64))
    stats = bb.merged_stats()
    sizes = [len(w.coords) for w in ws]
    print(json.dumps({
        "metric": "uneven batch G builds ms/batch (batched build: one launch per class, routed)",
        "value": round(m32_ms, 3), "unit": "ms/batch", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "higher_is_better": False, "data": "synthetic", "dtype": "f64 (routed units FP32)",
        "config": {"workload": f"c4: first {len(ws)} of 512 molecules, {min(sizes)}-{max(sizes)} atoms "
                               f"({sum(sizes)} atoms, {sum(w.n_ao for w in ws)} AO in all)"},
        "fp64_loop_ms": round(loop_ms, 3), "batched_fp64_ms": round(m64_ms, 3),
        "speedup_batched_routed_vs_fp64_loop": round(loop_ms / m32_ms, 4),
        "per_molecule_device_ms_fp64_loop": {"p50": round(float(np.percentile(per, 50)), 3),
                                             "p99": round(float(np.percentile(per, 99)), 3)},
        "max_abs_dG_batched_fp64_vs_loop": dG64, "max_abs_dG_batched_routed_vs_fp64": dG,
        "batched_learned_router_ms": round(mlp_ms, 3), "max_abs_dG_batched_learned_vs_fp64": dG_mlp,
        "router_training_quartets": n_tr,
        "class_launches_per_batch": stats["class_launches"], "work_units": stats["units"],
        "gpu_launches": 2 * stats["class_launches"] + 2,
        "host_plan_s": round(plan_s, 1)}))
    bb.close()


def reference_arm(a, rank, world):
    """The reference's CPU path on this host: the reference is pure Python
    (its host path at the workload's size is infeasible: the 6-atom c0 takes
    the times tests/golden/cpu_c0.npz records), so the arm runs its
    restatement, the oracle (oracle/oracle.c: the reference's eri_block over
    the plan's kept primitive pairs plus the six-block digest), on every host
    thread.  The quartets are the reference's own plan of the workload
    (tests/golden/plan_<workload>.npz, written by the reference's
    f_launches), screened by the reference's six-block rule; this library is
    not loaded.  Each of W + K steps is an independent timed sample (about
    12 s of CPU) extrapolated to one whole build; the value is the median
    over the K timed steps.  Rank 0 only."""
    if rank != 0:
        return
    from felizjueves_b200 import configs
    w = configs.by_name(a.workload)
    plan = reference_plan(a.workload)
    if plan is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no recorded reference plan for workload {a.workload}"}))
        return
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    times, spent = [], 0.0
    for i in range(a.warmup + a.steps):
        est, desc, cpu_s = cpu_estimate(w, plan, configs.perturbed_density(w.D, i % 20), cores,
                                        seed=i)
        spent += cpu_s
        if i >= a.warmup:
            times.append(est)
    wall = time.perf_counter() - t0
    v = float(np.median(times))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms/iter",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(v, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cluster, random symmetric densities)",
        "config": {"workload": WORKLOAD, "n_ao": w.n_ao, "shells": len(w.basis.shells),
                   "tau": w.tau},
        "estimate": "extrapolated: each step times a sample of the build's computed quartets "
                    "and scales it to the whole build; the build itself is not run",
        "sample_wall_s": round(wall, 1), "sample_cpu_s": round(spent, 1),
        "cpu_baseline": {"value": round(v, 1), "unit": "ms/iter", "cores": cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": round(v, 1), "unit": "ms/iter", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


if __name__ == "__main__":
    main()
