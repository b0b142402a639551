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
    ap.add_argument("--path", default="fock", choices=["fock", "coulomb", "df", "batch", "onee"],
                    help="fock: the G build (the headline); coulomb: the MMD J-engine; "
                         "df: DF-J/K (FP64 and split-BF16 tensor-core GEMMs); batch: the "
                         "uneven molecule batch (c4) as one captured graph")
    ap.add_argument("--molecules", type=int, default=64, help="batch path: the first N c4 molecules")
    ap.add_argument("--threshold", type=float, default=1e-9,
                    help="routed builds: the Schwarz x density bound under which a unit runs FP32 "
                         "(config c2's rule: 1e-9)")
    ap.add_argument("--budget-threshold", type=float, default=1e-7,
                    help="a second routed measurement at this threshold, reported with its "
                         "max|dG| against the 1e-8 budget (0: skip)")
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

def _time_quartets(args):
    """Worker (spawned): oracle eri_block + digest-free timing of quartets."""
    flat, quartets = args
    sys.path.insert(0, HERE)
    from oracle import oracle as O
    ob = O.OracleBasis(*flat)
    out = []
    for q in quartets:
        t = time.perf_counter()
        O.eri_block(ob, *q)
        out.append(time.perf_counter() - t)
    return out


def cpu_sample(w, lstats, plan, cores: int, budget_s: float = 15.0, seed: int = 0):
    """Estimated ms of the whole build on the oracle: per (class, K_AB, K_CD)
    launch key, time the oracle's ERI block on sampled computed-class
    quartets of that key; weight by the computed counts of the last GPU
    build.  A pilot of 2 quartets per key sets how many more each key gets
    so that the sampled CPU work comes to about `budget_s` seconds (at most
    200 per key).  Returns (ms_estimate, description, cpu_seconds_spent,
    wall_seconds)."""
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    keys = {}
    for li, s in enumerate(lstats):
        if s["computed"] == 0:
            continue
        k = (s["la"], s["lb"], s["lc"], s["ld"], s["kab"], s["kcd"])
        keys.setdefault(k, []).append(li)
    batches = plan.batches
    f = w.basis.flat()
    flat = (f["l"], f["centre"], f["prim0"], f["nprim"], f["exps"], f["coefs"])

    def draw(n_per):
        samples, owners = [], []
        for k, lis in sorted(keys.items()):
            for _ in range(n_per):
                L = plan.launches[lis[int(rng.integers(len(lis)))]]
                bp = batches[L.bra].pairs[int(rng.integers(len(batches[L.bra].pairs)))]
                kp = batches[L.ket].pairs[int(rng.integers(len(batches[L.ket].pairs)))]
                samples.append((bp.a, bp.b, kp.a, kp.b))
                owners.append(k)
        return samples, owners

    def run(samples, owners, per):
        chunks = [samples[i::cores] for i in range(cores)]
        with mp.get_context("spawn").Pool(cores) as pool:
            res = pool.map(_time_quartets, [(flat, c) for c in chunks])
        spent = 0.0
        for i in range(cores):
            for idx, t in zip(range(i, len(samples), cores), res[i]):
                per.setdefault(owners[idx], []).append(t)
                spent += t
        return spent

    per: dict = {}
    t0 = time.perf_counter()
    pilot = draw(2)
    spent = run(*pilot, per)
    n_more = int(min(200, max(0, 2 * (budget_s / max(spent, 1e-9) - 1))))
    n_samples = len(pilot[0])
    if n_more:
        more = draw(n_more)
        spent += run(*more, per)
        n_samples += len(more[0])
    wall = time.perf_counter() - t0
    total_cpu_s = 0.0
    for k, lis in keys.items():
        # the oracle sums every primitive pair of the sampled shells (no
        # pruning), so the estimate is an upper bound on the pruned work
        cnt = sum(lstats[li]["computed"] for li in lis)
        total_cpu_s += cnt * float(np.median(per[k]))
    ms = 1e3 * total_cpu_s / cores
    desc = (f"oracle eri_block (MMD, FP64) on {n_samples} sampled quartets, {2 + n_more} per "
            f"(class, K_AB, K_CD) key of the build's computed launches ({len(keys)} keys), median time "
            f"per key x computed quartets, summed, / {cores} core(s); {spent:.1f} s of CPU sampled; "
            f"digest not timed")
    return ms, desc, spent, wall


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
        router_info = install_learned_router(eng)
    budget = None
    if a.precision == "routed":
        ms, ck, nl, cs_r, ls_r, Gr = timed(_lib.FJB_ROUTED, a.threshold)
        n32, n64 = route_counts(eng)
        router_info = dict(router_info or {"kind": "bound"}, fp32_units=n32, fp64_units=n64)
        if a.budget_threshold > 0:
            msb, _, _, _, _, Gb = timed(_lib.FJB_ROUTED, a.budget_threshold)
            budget = {"threshold": a.budget_threshold, "ms_per_step": round(msb, 3),
                      "speedup_vs_fp64": round(ms64 / msb, 4),
                      "max_abs_dG_vs_fp64": float((Gb - G64).abs().max()),
                      "fp32_units": route_counts(eng)[0]}
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
    if not a.no_e2e and rank == 0:
        Dh = [configs.perturbed_density(w.D, i) for i in range(3)]
        eng.build_host(Dh[0], precision=prec, threshold=a.threshold)  # warm
        k2 = min(a.steps, 3)
        t0 = time.perf_counter()
        for i in range(k2):
            eng.build_host(Dh[i % 3], precision=prec, threshold=a.threshold)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / k2
        e2e = {"value": round(e2e_ms, 3), "unit": "ms/iter", "h2d_bytes_per_step": n * n * 8,
               "d2h_bytes_per_step": 3 * n * n * 8,
               "api": "fjb_fock_build_host (C ABI, host buffers; copies in the timed region)"}

    cpu = None
    if not a.no_cpu and rank == 0 and world == 1:
        cores = 1
        est, desc, spent, wall = cpu_sample(w, ls, P, cores)
        cpu = {"value": round(est, 1), "unit": "ms/iter", "cores": cores, "kind": "port",
               "sample": desc}

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
        "routed_at_budget_threshold": budget,
        "router": router_info,
        "config": {"workload": WORKLOAD, "n_ao": n, "shells": len(w.basis.shells),
                   "tau": w.tau, "quartets_launched": launched, "quartets_computed": computed,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "working set > 126 MB L2 (6 x 31.5 MB matrices + pair records); no flush"},
        "roofline": {"bound": "fp64", "kernel": "hgp_fock_kernel class (%d%d|%d%d)" % tcls,
                     "achieved": round(ach, 3), "peak": round(peak64, 3), "unit": "TFLOP/s",
                     "frac": round(ach / peak64, 4) if peak64 else None, "traffic": None,
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


def train_router():
    """The learned precision router: trained on the GPU with the library's
    kernels on quartets the FP64 method computes for six seeded 4-10 atom
    clusters (not a benchmarked system), calibrated on held-out quartets
    (0.999 residual quantile).  Returns (network, margin, training size)."""
    from felizjueves_b200 import configs, router
    X, y = router.training_set([configs.cluster(n, 100 + n) for n in (4, 5, 6, 7, 8, 10)], n_per=12000, seed=1)
    perm = np.random.default_rng(2).permutation(len(X))
    tr, va = perm[: int(0.8 * len(X))], perm[int(0.8 * len(X)):]
    mlp = router.MLP(router.init_params(X[tr], y[tr], seed=0))
    mlp.train(X[tr], y[tr])
    return mlp, router.calibrate(mlp, X[va], y[va], 0.999), int(len(tr))


def install_learned_router(eng) -> dict:
    """train_router(), installed on `eng` at the 1e-9 threshold."""
    from felizjueves_b200 import router
    mlp, margin, n_tr = train_router()
    router.install(eng, mlp, threshold=1e-9, margin=margin)
    return {"kind": "learned", "training_quartets": n_tr, "margin_log10": round(margin, 3)}


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
    if a.path == "coulomb":
        from felizjueves_b200.fock import FockEngine
        eng = FockEngine(w.basis, device=local)
        J = torch.empty_like(D)
        ms, _ = timed(lambda: eng.coulomb(D, tau=w.tau, J=J))
        line.update(metric="J-engine J build ms/iter", value=round(ms, 3), unit="ms/iter",
                    gpu_launches=eng.j_launches())
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
    else:
        from felizjueves_b200.df import DFEngine
        aux = configs.aux_basis(w)
        eng = DFEngine(w.basis, aux, device=local)
        B = eng.factors()
        ms64, (J64, K64) = timed(lambda: eng.jk(D, "fp64", B=B))
        ms16, (J16, K16) = timed(lambda: eng.jk(D, "bf16x3", B=B))
        line.update(metric="DF-J/K ms/iter", value=round(ms16, 3), unit="ms/iter", dtype="bf16x3 -> f32",
                    fp64_ms=round(ms64, 3), n_aux=aux.n_ao,
                    max_abs_dJ_bf16x3_vs_fp64=float((J16 - J64).abs().max()),
                    max_abs_dK_bf16x3_vs_fp64=float((K16 - K64).abs().max()))
    print(json.dumps(line))


def batch_path(a, local):
    """The c4 batch (its first --molecules molecules): the plain FP64
    per-molecule loop, the batch as one captured graph in FP64, and in the
    routed mode with the learned router (trained here on seeded 4-10 atom
    clusters, calibrated, installed on every molecule); total ms per batch,
    per-molecule device ms (p50, p99) and max|dG| against FP64."""
    import torch
    from felizjueves_b200 import _lib, configs, router
    from felizjueves_b200.batch import BatchBuilder
    torch.cuda.set_device(local)
    ws = configs.c4(a.molecules)
    bb = BatchBuilder(ws, device=local)
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
    bb.capture("fp64", _lib.FJB_FP64)
    g64_ms = timed(lambda: bb.replay("fp64"))
    G64 = [g.clone() for g in bb.G()]
    mlp, margin, _ = train_router()
    for eng in bb.engines:
        router.install(eng, mlp, threshold=1e-9, margin=margin)
    bb.capture("routed", _lib.FJB_ROUTED, 1e-9)
    gr_ms = timed(lambda: bb.replay("routed"))
    per = bb.device_ms()
    dG = max(float((g - h).abs().max()) for g, h in zip(bb.G(), G64))
    sizes = [len(w.coords) for w in ws]
    print(json.dumps({
        "metric": "uneven batch G builds ms/batch (one graph, routed + learned router)", "value": round(gr_ms, 3),
        "unit": "ms/batch", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "higher_is_better": False,
        "data": "synthetic", "dtype": "f64 (routed units FP32)",
        "config": {"workload": f"c4: first {len(ws)} of 512 molecules, {min(sizes)}-{max(sizes)} atoms "
                               f"({sum(sizes)} atoms, {sum(w.n_ao for w in ws)} AO in all)"},
        "fp64_loop_ms": round(loop_ms, 3), "fp64_graph_ms": round(g64_ms, 3),
        "per_molecule_device_ms": {"p50": round(float(np.percentile(per, 50)), 3),
                                   "p99": round(float(np.percentile(per, 99)), 3)},
        "max_abs_dG_vs_fp64": dG, "router_margin": round(margin, 3)}))


def reference_arm(a, rank, world):
    if rank != 0:
        return
    from felizjueves_b200 import configs
    from felizjueves_b200.fock import FockEngine
    w = configs.by_name(a.workload)
    # the plan is host work (no GPU); its launch counts come from the plan
    eng = FockEngine(w.basis, device=-1)
    P = eng.plan(w.D, w.tau, w.n_mag)
    ls = eng.launch_stats()
    # without a GPU build, every launched quartet is counted as computed:
    # the extrapolation is an upper bound on the CPU work of the screened
    # build by the fraction the six-block screen skips
    for s in ls:
        s["computed"] = s["launched"]
    cores = os.cpu_count() or 1
    times = []
    for i in range(max(1, a.warmup) + a.steps if a.steps <= 3 else 1 + min(a.steps, 3)):
        est, desc, spent, wall = cpu_sample(w, ls, P, cores, seed=i)
        times.append(est)
    v = float(np.median(times[1:] if len(times) > 1 else times))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms/iter",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(v, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD},
        "cpu_baseline": {"value": round(v, 1), "unit": "ms/iter", "cores": cores, "kind": "port",
                         "sample": desc + "; every launched quartet counted (no GPU screen)"},
        "e2e": {"value": round(v, 1), "unit": "ms/iter", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


if __name__ == "__main__":
    main()
