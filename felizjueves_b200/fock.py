"""The Fock build's host surface: the reference's driver-level API over the
C ABI of libfjb.so, with device memory and streams from PyTorch.

Mirrors (paths within the reference project):

* `f_launches(basis, D, *, tau, n)`  eri/fock/launch_f.py:390 -> FPlan,
  the pair stream as data (FPair, FBatch, FLaunch, counts()).  The bound is
  the reference's primitive_schwarz_bounds (ao/pairs.py:537), built in
  C++; it is not injectable here.
* `fock_two_electron(basis, D, *, tau, n)`  eri/fock/fock.py:166
  fock_two_electron_reference -> G = J - K/2, and
  `coulomb_exchange(basis, D, ...)`  eri/fock/fock.py:126 -> (J, K);
  `coulomb_matrix` (the J-engine, eri/j_coulomb/j.py:436) and
  `exchange_matrix` (eri/k_exchange/k.py:482) -> J or K alone.
* `eri_block(basis, a, b, c, d)`  eri/eri.py:145 -> the (ab|cd) block.
* `FockEngine`  the reusable form: plan once per (basis, tau, n), then build
  for any symmetric D, on device tensors (torch) or host arrays (numpy).
* `overlap_matrix`, `kinetic_matrix`, `potential_matrix`,
  `core_hamiltonian`, `FockEngine.one_electron`  the one-electron matrices
  the G build's caller needs (one_electron/overlap.py:67, kinetic.py:114,
  potential.py:101; H = T + V).

Refusals are the reference's: an asymmetric or non-finite D, a bad tau, an
l or a contraction degree above the compiled limits raise ValueError.  There
is no CPU path: every number comes from the sm_100a kernels.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Iterator

import numpy as np

from . import _lib
from .shell import Basis


@dataclass(frozen=True)
class FPair:
    a: int
    b: int
    la: int
    lb: int
    n_prim: int
    prims: tuple[int, ...]
    prim_G: tuple[float, ...]
    G: float
    dmax: float
    key: float
    mag: int

    @property
    def degree(self) -> int:
        return len(self.prims)


@dataclass(frozen=True)
class FBatch:
    la: int
    lb: int
    degree: int
    mag: int
    magnitude: float
    pairs: tuple[FPair, ...]

    @property
    def g_max(self) -> float:
        return max(p.G for p in self.pairs)


@dataclass(frozen=True)
class FLaunch:
    bra: int
    ket: int
    am: tuple[int, int, int, int]


@dataclass(frozen=True)
class FPlan:
    tau: float
    n: int
    magnitudes: tuple[float, ...]
    eps: float
    g_max: float
    batches: tuple[FBatch, ...]
    launches: tuple[FLaunch, ...]
    screened: tuple[tuple[int, int], ...]
    deleted: tuple[tuple[int, int], ...]
    n_prim_total: int
    quartets_launched: int = 0
    units: int = 0

    def __iter__(self) -> Iterator[FLaunch]:
        return iter(self.launches)

    def __len__(self) -> int:
        return len(self.launches)

    @property
    def pairs(self) -> tuple[FPair, ...]:
        return tuple(p for b in self.batches for p in b.pairs)

    @property
    def n_prim_kept(self) -> int:
        return sum(p.degree for p in self.pairs)

    def counts(self) -> dict[str, int]:
        nb = len(self.batches)
        return {"pairs": len(self.pairs) + len(self.deleted),
                "pairs_deleted": len(self.deleted),
                "primitive_pairs": self.n_prim_total,
                "primitive_pairs_pruned": self.n_prim_total - self.n_prim_kept,
                "batches": nb, "batch_pairs": nb * (nb + 1) // 2,
                "batch_pairs_screened": len(self.screened),
                "launches": len(self.launches)}


def _checked_density(basis: Basis, D) -> np.ndarray:
    n = basis.n_ao
    try:
        A = np.asarray(D, dtype=np.float64)
    except (TypeError, ValueError):
        raise ValueError(f"D is not an {n} x {n} matrix") from None
    if A.shape != (n, n):
        raise ValueError(f"D is not an {n} x {n} matrix")
    if not np.all(np.isfinite(A)):
        raise ValueError("D has a non-finite entry")
    if not np.array_equal(A, A.T):
        i, j = map(int, np.argwhere(A != A.T)[0])
        raise ValueError(f"D is not symmetric: D[{i}][{j}] = {A[i, j]!r} but "
                         f"D[{j}][{i}] = {A[j, i]!r}. An asymmetric density is "
                         "rejected, not symmetrised")
    return np.ascontiguousarray(A)


def _checked_tau(tau) -> float:
    import math
    if not (isinstance(tau, (int, float)) and not isinstance(tau, bool)
            and math.isfinite(tau) and tau >= 0.0):
        raise ValueError(f"tau = {tau!r} is not a finite float >= 0")
    return float(tau)


class FockEngine:
    """One basis on one GPU.  `plan(D, tau, n)` builds and stages the pair
    stream; `build(D)` runs the fused J/K/G build."""

    def __init__(self, basis: Basis, device: int = 0, tuned: bool = True):
        """`device` -1 makes a host-only handle (plans and lists, no builds);
        `tuned` applies the autotuner's shipped per-class configuration
        (felizjueves_b200/data/class_config.json) after each plan."""
        if not isinstance(basis, Basis):
            raise ValueError(f"{basis!r} is not a Basis")
        self.basis = basis
        self.device = int(device)
        self.tuned = bool(tuned)
        self._L = _lib.load()
        f = basis.flat()
        self._flat = f  # keep alive for the call
        bt = _lib.Basis_t(len(basis.shells), f["l"].ctypes.data, f["centre"].ctypes.data,
                          f["prim0"].ctypes.data, f["nprim"].ctypes.data,
                          f["exps"].ctypes.data, f["coefs"].ctypes.data)
        h = C.c_void_p()
        _lib.check(self._L.fjb_create(C.byref(h), C.byref(bt), self.device))
        self._h = h
        self._planned = False
        self._plan_lists = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.fjb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_ao(self) -> int:
        return self.basis.n_ao

    # -- the plan ----------------------------------------------------------
    def plan(self, D, tau: float = 1e-12, n: int = 4, *, export: bool = True) -> FPlan | None:
        """Plan the builds of density D: the pair stream on the host, staged
        on the device.  Returns the lists as an FPlan, or None with
        `export=False` (an SCF loop that only builds: the lists are then
        exported on first use)."""
        A = _checked_density(self.basis, D)
        tau = _checked_tau(tau)
        if type(n) is not int or n < 1:
            raise ValueError(f"n = {n!r} is not an int >= 1 (the number of eq. 29 magnitudes)")
        self._planned = False
        self._plan_lists = None
        _lib.check(self._L.fjb_plan(self._h, A.ctypes.data, tau, n), self._h)
        self._tau, self._n_mag, self._planned = tau, n, True
        if self.tuned and self.device >= 0:
            from . import autotune
            table = autotune.load_default()
            if table:
                autotune.apply(self, table)
        return self._plan if export else None

    @property
    def _plan(self) -> FPlan | None:
        """The current plan's lists (exported from the handle once)."""
        if not self._planned:
            return None
        if self._plan_lists is None:
            self._plan_lists = self._export(self._n_mag)
        return self._plan_lists

    def counts_raw(self) -> dict[str, int]:
        c = _lib.PlanCounts_t()
        _lib.check(self._L.fjb_plan_counts(self._h, C.byref(c)), self._h)
        return {k: int(getattr(c, k)) for k, _ in c._fields_}

    def _export(self, n: int) -> FPlan:
        c = self.counts_raw()
        nb, nk, npr = c["batches"], c["kept_pairs"], c["kept_prims"]
        arr = {
            "batch_key": np.zeros(4 * nb, np.int32), "batch_npairs": np.zeros(nb, np.int32),
            "pair_ab": np.zeros(2 * nk, np.int32), "pair_mag": np.zeros(nk, np.int32),
            "prims": np.zeros(npr, np.int32), "pair_G": np.zeros(nk), "pair_dmax": np.zeros(nk),
            "pair_key": np.zeros(nk), "prim_G": np.zeros(npr),
            "launches": np.zeros(2 * c["launches"], np.int32),
            "screened": np.zeros(2 * c["batch_pairs_screened"], np.int32),
            "deleted": np.zeros(2 * c["pairs_deleted"], np.int32),
            "magnitudes": np.zeros(n), "eps": np.zeros(1), "g_max": np.zeros(1)}
        lists = _lib.PlanLists_t(**{k: v.ctypes.data for k, v in arr.items()})
        _lib.check(self._L.fjb_plan_export(self._h, C.byref(lists)), self._h)
        shells = self.basis.shells
        bk = arr["batch_key"].reshape(-1, 4)
        pab = arr["pair_ab"].reshape(-1, 2)
        batches, ip, ik = [], 0, 0
        mags = tuple(float(x) for x in arr["magnitudes"])
        for bi in range(nb):
            la, lb, deg, mag = map(int, bk[bi])
            pairs = []
            for _ in range(int(arr["batch_npairs"][bi])):
                a, b = map(int, pab[ip])
                pairs.append(FPair(a, b, la, lb, shells[a].n_prim * shells[b].n_prim,
                                   tuple(int(x) for x in arr["prims"][ik:ik + deg]),
                                   tuple(float(x) for x in arr["prim_G"][ik:ik + deg]),
                                   float(arr["pair_G"][ip]), float(arr["pair_dmax"][ip]),
                                   float(arr["pair_key"][ip]), int(arr["pair_mag"][ip])))
                ip += 1
                ik += deg
            batches.append(FBatch(la, lb, deg, mag, mags[mag], tuple(pairs)))
        L = arr["launches"].reshape(-1, 2)
        launches = tuple(FLaunch(int(i), int(j), (batches[i].la, batches[i].lb,
                                                  batches[j].la, batches[j].lb))
                         for i, j in L)
        return FPlan(self._tau, n, mags, float(arr["eps"][0]),
                     float(arr["g_max"][0]), tuple(batches), launches,
                     tuple(map(tuple, arr["screened"].reshape(-1, 2).tolist())),
                     tuple(map(tuple, arr["deleted"].reshape(-1, 2).tolist())),
                     c["primitive_pairs"], c["quartets_launched"], c["units"])

    # -- builds --------------------------------------------------------------
    def _require_plan(self):
        if not self._planned:
            raise RuntimeError("no plan: call plan(D, tau, n) first")

    def build(self, D, *, J=None, K=None, G=None, precision: int = _lib.FJB_FP64,
              threshold: float = 0.0, stream=None, graph: bool = False):
        """Device build: D (torch, cuda, float64, n x n, symmetric) in; J, K,
        G (allocated if not given) out.  Stream-ordered, not synchronised.
        `graph=True` replays the build as a captured CUDA graph (captured on
        the first call for these tensors; update D in place between calls)."""
        import torch
        self._require_plan()
        n = self.n_ao
        if not (isinstance(D, torch.Tensor) and D.is_cuda and D.dtype == torch.float64
                and tuple(D.shape) == (n, n) and D.is_contiguous()):
            raise ValueError(f"D must be a contiguous cuda float64 tensor of shape ({n}, {n})")
        out = []
        for M in (J, K, G):
            if M is None:
                M = torch.empty((n, n), dtype=torch.float64, device=D.device)
            out.append(M)
        st = stream if stream is not None else torch.cuda.current_stream(D.device)
        fn = self._L.fjb_fock_build_graph if graph else self._L.fjb_fock_build
        _lib.check(fn(self._h, D.data_ptr(), out[0].data_ptr(), out[1].data_ptr(),
                      out[2].data_ptr(), int(precision), float(threshold),
                      C.c_void_p(st.cuda_stream)), self._h)
        return tuple(out)

    def set_rys(self, mode=1) -> None:
        """Which classes the Rys kernel takes (fjb_set_rys): 1 or True (the
        default) the large classes, 0 or False none (the HGP interpreter),
        2 every class it has."""
        _lib.check(self._L.fjb_set_rys(self._h, int(mode)), self._h)

    def set_route_check(self, budget: float = 1e-8, stride: int = 32) -> None:
        """The routed build's error-budget check (fjb_set_route_check): a
        sampled FP64 re-build of every stride-th FP32 unit estimates the
        FP32 error in G; over `budget` the build re-runs its FP32 units in
        FP64.  budget <= 0 turns it off."""
        _lib.check(self._L.fjb_set_route_check(self._h, float(budget), int(stride)), self._h)

    def route_check(self) -> tuple[float, bool]:
        """(estimated max|dG| of the FP32 units, re-routed to FP64?) of the
        last routed build."""
        est, flag = C.c_double(), C.c_int()
        _lib.check(self._L.fjb_route_check_result(self._h, C.byref(est), C.byref(flag)), self._h)
        return float(est.value), bool(flag.value)

    def build_host(self, D, *, precision: int = _lib.FJB_FP64, threshold: float = 0.0, out=None):
        """Host build through the C ABI's host-buffer entry point: numpy in,
        (J, K, G) numpy out -- into `out`, three C-contiguous float64 n x n
        arrays (e.g. views of pinned host memory), when given."""
        self._require_plan()
        A = _checked_density(self.basis, D)
        n = self.n_ao
        if out is None:
            J, K, G = (np.empty((n, n)) for _ in range(3))
        else:
            J, K, G = out
            for M in out:
                if not (isinstance(M, np.ndarray) and M.dtype == np.float64 and M.shape == (n, n)
                        and M.flags.c_contiguous):
                    raise ValueError(f"out: three C-contiguous float64 {n} x {n} arrays")
        _lib.check(self._L.fjb_fock_build_host(self._h, A.ctypes.data, J.ctypes.data,
                                               K.ctypes.data, G.ctypes.data,
                                               int(precision), float(threshold)), self._h)
        return J, K, G

    def scatter_map(self, launch: int) -> dict[str, np.ndarray]:
        """The atomics-free build's map of plan launch `launch`
        (eri/fock/kernel_f_scatter.py:203-260 scatter_map): `el` (n_el x 2,
        (row, col) ascending), `ptr` (n_el + 1), `src` (each element's slots
        ascending, in the reference's slot layout)."""
        self._require_plan()
        ne, ns = C.c_int64(), C.c_int64()
        _lib.check(self._L.fjb_scatter_map(self._h, int(launch), None, None, None, C.byref(ne),
                                           C.byref(ns)), self._h)
        el = np.empty(2 * ne.value, np.int32)
        ptr = np.empty(ne.value + 1, np.int32)
        src = np.empty(ns.value, np.int32)
        _lib.check(self._L.fjb_scatter_map(self._h, int(launch), el.ctypes.data, ptr.ctypes.data,
                                           src.ctypes.data, C.byref(ne), C.byref(ns)), self._h)
        return {"el": el.reshape(-1, 2), "ptr": ptr, "src": src}

    # -- the J-engine (eri/j_coulomb/j.py) ----------------------------------
    def coulomb(self, D, *, tau: float = 0.0, J=None, threshold: float = 0.0):
        """J of the symmetric density D by the McMurchie-Davidson J-engine
        (the reference's coulomb_matrix / coulomb_matrix_screened sweep,
        eri/j_coulomb/j.py:436-581): a device tensor D in, a device J out
        (written in full).  Needs no plan.  threshold > 0: the FP32 E/R tier
        for record pairs whose bound is under it (fjb_coulomb_mixed)."""
        import torch
        tau = _checked_tau(tau)
        if not isinstance(D, torch.Tensor):
            D = torch.as_tensor(_checked_density(self.basis, D), device=f"cuda:{self.device}")
        n = self.n_ao
        if D.shape != (n, n) or D.dtype != torch.float64 or not D.is_contiguous():
            raise ValueError(f"D must be a contiguous float64 ({n}, {n}) tensor")
        if J is None:
            J = torch.empty_like(D)
        st = torch.cuda.current_stream(D.device).cuda_stream
        _lib.check(self._L.fjb_coulomb_mixed(self._h, D.data_ptr(), J.data_ptr(), tau, float(threshold),
                                             C.c_void_p(st)), self._h)
        return J

    # -- the one-electron matrices (one_electron/) ---------------------------
    def one_electron(self, nuclei, *, S=None, T=None, V=None, H=None, want=("S", "T", "V", "H")):
        """(S, T, V, H) of the basis as device tensors (H = T + V, the core
        Hamiltonian), for nuclei [(Z, (x, y, z)), ...] in Bohr
        (one_electron/overlap.py, kinetic.py, potential.py; potential.py's
        Nucleus).  Matrices not in `want` are not computed into and come
        back None; given tensors are written in full.  Needs no plan."""
        import torch
        nuc = _checked_nuclei(nuclei)
        charges = np.ascontiguousarray([z for z, _ in nuc], np.float64)
        coords = np.ascontiguousarray([c for _, c in nuc], np.float64).reshape(-1)
        n = self.n_ao
        dev = torch.device(f"cuda:{self.device}")
        out = []
        for name, M in (("S", S), ("T", T), ("V", V), ("H", H)):
            if name not in want:
                out.append(None)
                continue
            if M is None:
                M = torch.empty((n, n), dtype=torch.float64, device=dev)
            elif not (M.is_cuda and M.dtype == torch.float64 and tuple(M.shape) == (n, n) and M.is_contiguous()):
                raise ValueError(f"{name} must be a contiguous cuda float64 ({n}, {n}) tensor")
            out.append(M)
        st = torch.cuda.current_stream(dev).cuda_stream
        ptr = [None if M is None else M.data_ptr() for M in out]
        _lib.check(self._L.fjb_one_electron(self._h, charges.ctypes.data if len(nuc) else None,
                                            coords.ctypes.data if len(nuc) else None, len(nuc), *ptr,
                                            C.c_void_p(st)), self._h)
        return tuple(out)

    def j_launches(self) -> int:
        """Kernel launches of the last `coulomb` call."""
        return int(self._L.fjb_j_last_launches(self._h))

    def j_plan_lists(self, D) -> dict[str, np.ndarray]:
        """The J-engine's host plan for D (eri/j_coulomb/launch.py:274-327):
        per record (sweep order) its shell pair a >= b, primitive index, L,
        I_pair and ket key; `ket_order` the records sorted descending by key
        per L (stable), `L_off` the offsets of each L in it."""
        A = _checked_density(self.basis, D)
        n = C.c_int64()
        _lib.check(self._L.fjb_j_plan_lists(self._h, A.ctypes.data, None, C.byref(n)), self._h)
        m = int(n.value)
        out = {k: np.empty(m, np.int32) for k in ("a", "b", "prim", "L", "ket_order")}
        out.update(G=np.empty(m), key=np.empty(m), L_off=np.empty(8, np.int64))
        lst = _lib.JLists_t(*(out[k].ctypes.data for k in ("a", "b", "prim", "L", "G", "key",
                                                             "ket_order", "L_off")))
        _lib.check(self._L.fjb_j_plan_lists(self._h, A.ctypes.data, C.byref(lst), C.byref(n)), self._h)
        return out

    def last_build_stats(self) -> tuple[float, int]:
        ms, nl = C.c_double(), C.c_int()
        _lib.check(self._L.fjb_last_build_stats(self._h, C.byref(ms), C.byref(nl)), self._h)
        return float(ms.value), int(nl.value)

    def set_class_config(self, cls, threads: int = 0, slots: int = 0) -> None:
        """CTA width and primitive-quartet chunk of one class (0 = default)."""
        _lib.check(self._L.fjb_set_class_config(self._h, *map(int, cls), int(threads),
                                                int(slots)), self._h)

    def set_class_config32(self, cls, threads: int = 0, slots: int = 0) -> None:
        """The same for the routed path's FP32 interpreter kernel of a class
        (0, 0 = the FP64 configuration's FP32 twin)."""
        _lib.check(self._L.fjb_set_class_config32(self._h, *map(int, cls), int(threads),
                                                  int(slots)), self._h)

    def plan_units(self) -> np.ndarray:
        """The plan's work units, (n, 4) int32 rows (launch, bra pair
        index, first ket, end ket), in the order the class kernels take
        them (fjb_plan_units)."""
        n = C.c_int64()
        _lib.check(self._L.fjb_plan_units(self._h, None, 0, C.byref(n)), self._h)
        out = np.zeros((max(n.value, 1), 4), np.int32)
        _lib.check(self._L.fjb_plan_units(self._h, out.ctypes.data, n.value, C.byref(n)), self._h)
        return out[: n.value]

    def launch_stats(self) -> list[dict]:
        """Per launch: class, degrees, quartets met and computed by the last
        build."""
        n = self.counts_raw()["launches"]
        arr = (_lib.LaunchStat_t * max(n, 1))()
        _lib.check(self._L.fjb_launch_stats(self._h, C.cast(arr, C.c_void_p), n), self._h)
        return [{k: getattr(arr[i], k) for k, _ in _lib.LaunchStat_t._fields_} for i in range(n)]

    def class_stats(self) -> list[dict]:
        """Per class kernel of the last build: class, ms, work units."""
        nc = C.c_int64()
        _lib.check(self._L.fjb_class_stats(self._h, None, 0, C.byref(nc)), self._h)
        arr = (_lib.ClassStat_t * max(nc.value, 1))()
        _lib.check(self._L.fjb_class_stats(self._h, C.cast(arr, C.c_void_p), nc.value,
                                           C.byref(nc)), self._h)
        return [{k: getattr(arr[i], k) for k, _ in _lib.ClassStat_t._fields_}
                for i in range(nc.value)]

    # --- the split build's ordered pair stream (eri/hjk/launch_hjk.py) -----

    HJK_MODES = {"ordered": 0, "canonical": 1}
    HJK_SCREENS = {"j": 0, "k": 1}

    def hjk_plan(self, D, tau: float = 1e-12, *, mode: str = "ordered", screen: str = "k") -> dict:
        """The split build's stream (fjb_hjk_plan; `hjk_launches`): every
        ordered shell pair, bins (la, lb, degree), every ordered batch pair
        a launch.  Returns its lists as arrays: `pairs` (a, b, la, lb,
        degree) in batch order, `pair_G`, `batches` (la, lb, degree, first
        pair, pairs), `launches` (bra, ket, ordered class, kernel class,
        shells), and `counts` (pairs, batches, launches, classes, quartets,
        quartets_skipped)."""
        if mode not in self.HJK_MODES:
            raise ValueError(f"mode = {mode!r} is not one of {tuple(self.HJK_MODES)}")
        if screen not in self.HJK_SCREENS:
            raise ValueError(f"screen = {screen!r} is not one of {tuple(self.HJK_SCREENS)}")
        Dh = _checked_density(self.basis, D)
        _lib.check(self._L.fjb_hjk_plan(self._h, Dh.ctypes.data, float(tau), self.HJK_MODES[mode],
                                        self.HJK_SCREENS[screen]), self._h)
        cnt = np.zeros(6, np.int64)
        _lib.check(self._L.fjb_hjk_counts(self._h, cnt.ctypes.data), self._h)
        n_p, n_b, n_l = int(cnt[0]), int(cnt[1]), int(cnt[2])
        pairs = np.zeros((n_p, 5), np.int32)
        pair_G = np.zeros(n_p)
        batches = np.zeros((n_b, 5), np.int32)
        launches = np.zeros((n_l, 14), np.int32)
        _lib.check(self._L.fjb_hjk_export(self._h, pairs.ctypes.data, pair_G.ctypes.data, batches.ctypes.data,
                                          launches.ctypes.data), self._h)
        names = ("pairs", "batches", "launches", "classes", "quartets", "quartets_skipped")
        return {"pairs": pairs, "pair_G": pair_G, "batches": batches, "launches": launches,
                "counts": dict(zip(names, map(int, cnt)))}

    def hjk_keys(self, launch: int, n_visits: int) -> tuple[np.ndarray, np.ndarray]:
        """One launch's visit keys and skip flags (bra pair outer)."""
        keys = np.zeros(n_visits)
        skipped = np.zeros(n_visits, np.uint8)
        _lib.check(self._L.fjb_hjk_keys(self._h, int(launch), keys.ctypes.data, skipped.ctypes.data), self._h)
        return keys, skipped.astype(bool)

    def hjk_k(self, D, K=None, stream=None):
        """K over the split stream (fjb_hjk_k): every ordered quartet not
        skipped by K's key deposits K[a][c] += D[b][d] (ab|cd)."""
        import torch
        if K is None:
            K = torch.empty_like(D)
        st = stream if stream is not None else torch.cuda.current_stream(D.device)
        _lib.check(self._L.fjb_hjk_k(self._h, D.data_ptr(), K.data_ptr(), C.c_void_p(st.cuda_stream)), self._h)
        return K

    def hjk_computed(self, n_launches: int) -> np.ndarray:
        """Per launch, the quartets the last hjk_k computed on the device."""
        out = np.zeros(n_launches, np.int64)
        _lib.check(self._L.fjb_hjk_computed(self._h, out.ctypes.data), self._h)
        return out

    def screen_mask(self, D, at=None) -> np.ndarray:
        """Per launched quartet (launch, bra pair, ket pair order), 1 when
        the six-block screen skips it (walk_f.py:344-380); only the entries
        at positions `at` (gathered on the device) when given."""
        import torch
        self._require_plan()
        Dt = torch.as_tensor(_checked_density(self.basis, D if not hasattr(D, "cpu") else D.cpu().numpy()),
                             device=f"cuda:{self.device}")
        m = torch.zeros(self._plan.quartets_launched, dtype=torch.uint8, device=Dt.device)
        _lib.check(self._L.fjb_screen_mask(self._h, Dt.data_ptr(), m.data_ptr(),
                                           C.c_void_p(torch.cuda.current_stream(Dt.device).cuda_stream)),
                   self._h)
        torch.cuda.synchronize(Dt.device)
        if at is not None:
            m = m[torch.as_tensor(np.asarray(at, np.int64), device=Dt.device)]
        return m.cpu().numpy()

    def eri_blocks(self, quartets, fp32: bool = False) -> list[np.ndarray]:
        """(ab|cd) of ordered shell quartets, each a (n_a n_b, n_c n_d) array
        in the reference's eri_block layout; `fp32` with the routed path's
        FP32 recurrences (what a quartet routed to FP32 contributes)."""
        import torch
        q = np.ascontiguousarray(np.asarray(quartets, np.int32).reshape(-1, 4))
        off = np.zeros(len(q) + 1, np.int64)
        sizes = [np.prod([self.basis.shells[s].n_cart for s in row]) for row in q]
        total = int(np.sum(sizes)) if len(q) else 0
        out = torch.zeros(max(total, 1), dtype=torch.float64, device=f"cuda:{self.device}")
        fn = self._L.fjb_eri_blocks_fp32 if fp32 else self._L.fjb_eri_blocks
        _lib.check(fn(self._h, q.ctypes.data, len(q), out.data_ptr(), off.ctypes.data), self._h)
        flat = out.cpu().numpy()
        res = []
        for i, row in enumerate(q):
            na, nb, nc, nd = (self.basis.shells[s].n_cart for s in row)
            res.append(flat[off[i]:off[i + 1]].reshape(na * nb, nc * nd))
        return res


def f_launches(basis: Basis, D, *, tau: float, n: int, device: int = 0) -> FPlan:
    eng = FockEngine(basis, device)
    return eng.plan(D, tau, n)


def _checked_nuclei(nuclei) -> list[tuple[float, tuple[float, float, float]]]:
    """Nuclei as [(Z, (x, y, z))], refused as the reference's _check_nuclei
    does (one_electron/potential.py:67-76)."""
    out = []
    for nu in nuclei:
        if len(nu) != 2:
            raise ValueError(f"nucleus {nu!r} is not (Z, centre)")
        Z, c = nu
        if len(c) != 3:
            raise ValueError(f"nucleus centre {c!r} is not three coordinates")
        nz = (float(Z), (float(c[0]), float(c[1]), float(c[2])))
        if not all(np.isfinite([nz[0], *nz[1]])):
            raise ValueError(f"nucleus {nu!r} has a non-finite charge or coordinate")
        out.append(nz)
    return out


def overlap_matrix(basis: Basis, *, device: int = 0) -> np.ndarray:
    """S (one_electron/overlap.py:67), on the GPU."""
    return FockEngine(basis, device).one_electron([], want=("S",))[0].cpu().numpy()


def kinetic_matrix(basis: Basis, *, device: int = 0) -> np.ndarray:
    """T (one_electron/kinetic.py:114), on the GPU."""
    return FockEngine(basis, device).one_electron([], want=("T",))[1].cpu().numpy()


def potential_matrix(basis: Basis, nuclei, *, device: int = 0) -> np.ndarray:
    """V = -sum_C Z_C <a|1/r_C|b> (one_electron/potential.py:101), on the GPU."""
    return FockEngine(basis, device).one_electron(nuclei, want=("V",))[2].cpu().numpy()


def core_hamiltonian(basis: Basis, nuclei, *, device: int = 0) -> np.ndarray:
    """H = T + V, on the GPU."""
    return FockEngine(basis, device).one_electron(nuclei, want=("H",))[3].cpu().numpy()


def coulomb_exchange(basis: Basis, D, *, tau: float = 0.0, n: int = 4, device: int = 0):
    """(J, K) of the total density D (numpy arrays), on the GPU."""
    eng = FockEngine(basis, device)
    eng.plan(D, tau, n, export=False)
    J, K, _ = eng.build_host(D)
    return J, K


def fock_two_electron(basis: Basis, D, *, tau: float = 0.0, n: int = 4, device: int = 0):
    """G = J - K/2 of the total closed-shell density D, on the GPU."""
    eng = FockEngine(basis, device)
    eng.plan(D, tau, n, export=False)
    return eng.build_host(D)[2]


def coulomb_matrix(basis: Basis, D, *, tau: float = 0.0, device: int = 0) -> np.ndarray:
    """J_mn of the symmetric density D (numpy) by the J-engine on the GPU:
    the reference's coulomb_matrix (eri/j_coulomb/j.py:436-450) at tau = 0,
    its screened sweep (j.py:538-581) at tau > 0."""
    import torch
    eng = FockEngine(basis, device)
    Dt = torch.as_tensor(_checked_density(basis, D), device=f"cuda:{device}")
    J = eng.coulomb(Dt, tau=tau)
    torch.cuda.synchronize(Dt.device)
    return J.cpu().numpy()


def exchange_matrix(basis: Basis, D, *, tau: float = 0.0, n: int = 4, device: int = 0) -> np.ndarray:
    """K_ab = sum_cd D_cd (ac|bd) of the symmetric density D (numpy), on the
    GPU: the reference's exchange_matrix (eri/k_exchange/k.py:482; its
    staged MMD sweep) computed by the fused build, whose K is the same sum
    over the 8-fold orbits (unscreened at tau = 0)."""
    eng = FockEngine(basis, device)
    eng.plan(D, tau, n, export=False)
    return eng.build_host(D)[1]


def eri_block(basis: Basis, a: int, b: int, c: int, d: int, device: int = 0) -> np.ndarray:
    return FockEngine(basis, device).eri_blocks([(a, b, c, d)])[0]


def diagonal_matrix(basis: Basis, device: int = 0) -> np.ndarray:
    """(mn|mn) for every AO pair, n_ao x n_ao (eri/schwarz.py:86-93): the
    diagonals of the (ab|ab) blocks of every shell pair a <= b, computed on
    the GPU by the build's own HGP recurrences, placed at (m, n) and (n, m)."""
    sh, off = basis.shells, basis.offsets
    quartets = [(a, b, a, b) for a in range(len(sh)) for b in range(a, len(sh))]
    blocks = FockEngine(basis, device, tuned=False).eri_blocks(quartets)
    M = np.zeros((basis.n_ao, basis.n_ao))
    for (a, b, _, _), blk in zip(quartets, blocks):
        na, nb = sh[a].n_cart, sh[b].n_cart
        d = np.diagonal(blk).reshape(na, nb)
        M[off[a]:off[a] + na, off[b]:off[b] + nb] = d
        M[off[b]:off[b] + nb, off[a]:off[a] + na] = d.T
    return M


def schwarz_matrix(basis: Basis, device: int = 0) -> np.ndarray:
    """Q[m][n] = sqrt(max((mn|mn), 0)), symmetric (eri/schwarz.py:102)."""
    return np.sqrt(np.maximum(diagonal_matrix(basis, device), 0.0))
