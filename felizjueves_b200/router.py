"""The learned precision router: training data from the FP64 method, GPU
training with the library's own kernels, calibration, installation.

The network (csrc/router.cuh) maps 12 pair features of a quartet to the
predicted log10 of its largest deposit into G, max|(ab|cd)| x dmax (dmax the
six-block weighted density maximum the screen reads), as the log10 Schwarz x
density bound (a fixed skip term) plus a learned gap below it.  Training targets are
computed by the FP64 method itself: the ERI blocks of sampled launched
quartets from the HGP tap (`FockEngine.eri_blocks`).  Training runs on the
GPU: `fjb_mlp_gradient` (forward + backward) and `fjb_mlp_adam`, mini-batch
Adam on the mean squared error.

Routing is conservative by construction: a unit of work goes to FP32 only
when every computed quartet of it is under the rigorous Schwarz x density
bound, or predicted under the threshold after subtracting a calibrated
margin (a high quantile of the validation residuals y - y_pred).  Skipping is
never the router's: the six-block screen decides it.  `validate` builds the
routed and the FP64 G once and turns the learned router off if the
difference breaks the error budget (the FP64 fallback).
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .fock import FockEngine

N_FEAT = 12


def n_params() -> int:
    return int(_lib.load().fjb_mlp_n_params())


def init_params(X: np.ndarray, y: np.ndarray | None = None, seed: int = 0) -> np.ndarray:
    """mu, sd from the training features; Glorot-scaled random weights; the
    output bias at the mean gap y - bound of the training targets (when
    given), so training starts from "deposit = bound x typical gap"."""
    rng = np.random.default_rng(seed)
    mu = X.mean(0)
    sd = X.std(0)
    sd[sd < 1e-3] = 1.0
    W1 = rng.normal(0, 1 / math.sqrt(N_FEAT), (64, N_FEAT))
    W2 = rng.normal(0, 1 / math.sqrt(64), (64, 64))
    w3 = rng.normal(0, 0.1 / math.sqrt(64), 64)
    b3 = 0.0 if y is None else float(np.mean(y - bound_log10(X)))
    p = np.concatenate([mu, sd, W1.ravel(), np.zeros(64), W2.ravel(), np.zeros(64), w3, [b3]])
    assert p.size == n_params()
    return p.astype(np.float32)


def bound_log10(X: np.ndarray) -> np.ndarray:
    """log10 of the Schwarz x density bound of each sample (features 9-11),
    the fixed skip term of the network's output."""
    return X[:, 9:12].astype(np.float64).sum(1)


class MLP:
    """Parameters and Adam state on the device."""

    def __init__(self, params: np.ndarray, device: int = 0):
        import torch
        self.dev = torch.device(f"cuda:{device}")
        self.p = torch.tensor(params, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step = 0
        self._L = _lib.load()

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy()

    def predict(self, X, *, exact: bool = False):
        """The network's prediction in the routing pass's own arithmetic
        (fjb_mlp_forward_tc: FP16 tensor-core products), or with `exact` in
        the FP32 arithmetic of training (fjb_mlp_forward)."""
        import torch
        X = torch.as_tensor(X, dtype=torch.float32, device=self.dev).contiguous()
        Y = torch.empty(len(X), dtype=torch.float32, device=self.dev)
        f = self._L.fjb_mlp_forward if exact else self._L.fjb_mlp_forward_tc
        _lib.check(f(self.p.data_ptr(), X.data_ptr(), len(X), Y.data_ptr(), None))
        return Y

    def gradient(self, X, T):
        """(gradient, mean squared error) of one batch, by the library's
        kernels."""
        import torch
        X = torch.as_tensor(X, dtype=torch.float32, device=self.dev).contiguous()
        T = torch.as_tensor(T, dtype=torch.float32, device=self.dev).contiguous()
        n = len(X)
        g = torch.zeros_like(self.p)
        se = torch.empty(n, dtype=torch.float32, device=self.dev)
        scratch = torch.empty(n * 257, dtype=torch.float32, device=self.dev)
        _lib.check(self._L.fjb_mlp_gradient(self.p.data_ptr(), X.data_ptr(), T.data_ptr(), n,
                                            g.data_ptr(), se.data_ptr(), scratch.data_ptr(), None))
        return g, float(se.mean())

    def train(self, X, T, *, epochs: int = 60, batch: int = 2048, lr: float = 3e-3,
              seed: int = 0) -> list[float]:
        """Mini-batch Adam on the mean squared error in log10 units, the
        learning rate halved every third of the epochs.  Returns the
        per-epoch mean squared error."""
        import torch
        rng = np.random.default_rng(seed)
        X = torch.as_tensor(X, dtype=torch.float32, device=self.dev)
        T = torch.as_tensor(T, dtype=torch.float32, device=self.dev)
        n = len(X)
        losses = []
        for ep in range(epochs):
            rate = lr * 0.5 ** (3 * ep // max(epochs, 1))
            perm = torch.as_tensor(rng.permutation(n), device=self.dev)
            tot = 0.0
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch]
                g, mse = self.gradient(X[idx], T[idx])
                self.step += 1
                _lib.check(self._L.fjb_mlp_adam(self.p.data_ptr(), g.data_ptr(), self.m.data_ptr(),
                                                self.v.data_ptr(), C.c_float(rate), self.step, None))
                tot += mse * len(idx)
            losses.append(tot / n)
        return losses


def plan_samples(eng: FockEngine, n: int, rng) -> tuple[np.ndarray, np.ndarray]:
    """n random launched quartets as (launch, bra index, ket index) and their
    shells (a, b, c, d), drawn like sample_launched but from the handle's
    exported arrays, vectorised (no per-pair objects: 64-atom plans)."""
    c = eng.counts_raw()
    nb, nk, nl = c["batches"], c["kept_pairs"], c["launches"]
    arr = {"batch_key": np.zeros(4 * nb, np.int32), "batch_npairs": np.zeros(nb, np.int32),
           "pair_ab": np.zeros(2 * nk, np.int32), "pair_mag": np.zeros(nk, np.int32),
           "prims": np.zeros(c["kept_prims"], np.int32), "pair_G": np.zeros(nk), "pair_dmax": np.zeros(nk),
           "pair_key": np.zeros(nk), "prim_G": np.zeros(c["kept_prims"]),
           "launches": np.zeros(2 * nl, np.int32),
           "screened": np.zeros(2 * c["batch_pairs_screened"], np.int32),
           "deleted": np.zeros(2 * c["pairs_deleted"], np.int32),
           "magnitudes": np.zeros(eng._n_mag), "eps": np.zeros(1), "g_max": np.zeros(1)}
    lists = _lib.PlanLists_t(**{k: v.ctypes.data for k, v in arr.items()})
    _lib.check(eng._L.fjb_plan_export(eng._h, C.byref(lists)), eng._h)
    npairs = arr["batch_npairs"].astype(np.int64)
    p0 = np.concatenate([[0], np.cumsum(npairs)[:-1]])
    L = arr["launches"].reshape(-1, 2)
    sizes = (npairs[L[:, 0]] * npairs[L[:, 1]]).astype(np.float64)
    li = rng.choice(nl, size=n, p=sizes / sizes.sum())
    ib = (rng.random(n) * npairs[L[li, 0]]).astype(np.int64)
    ik = (rng.random(n) * npairs[L[li, 1]]).astype(np.int64)
    diag = (L[li, 0] == L[li, 1]) & (ik < ib)
    ib[diag], ik[diag] = ik[diag], ib[diag].copy()
    ab = arr["pair_ab"].reshape(-1, 2)
    bra, ket = ab[p0[L[li, 0]] + ib], ab[p0[L[li, 1]] + ik]
    samples = np.stack([li, ib, ik], axis=1).astype(np.int32)
    return samples, np.concatenate([bra, ket], axis=1).astype(np.int32)


def sample_launched(eng: FockEngine, n: int, rng) -> np.ndarray:
    """n random launched quartets (launch, bra index, ket index), launches
    drawn by the quartets they hold; the canonical half on the diagonal."""
    P = eng._plan
    sizes = np.array([len(P.batches[L.bra].pairs) * len(P.batches[L.ket].pairs) for L in P.launches],
                     np.float64)
    li = rng.choice(len(P.launches), size=n, p=sizes / sizes.sum())
    out = np.empty((n, 3), np.int32)
    for k, l in enumerate(li):
        L = P.launches[l]
        nb, nk = len(P.batches[L.bra].pairs), len(P.batches[L.ket].pairs)
        ib, ik = int(rng.integers(nb)), int(rng.integers(nk))
        if L.bra == L.ket and ik < ib:
            ib, ik = ik, ib
        out[k] = (l, ib, ik)
    return out


def features(eng: FockEngine, D, samples: np.ndarray):
    """Device features (n x 12) and six-block bounds of sampled quartets."""
    import torch
    n = len(samples)
    Dt = torch.as_tensor(np.ascontiguousarray(D, np.float64), device=f"cuda:{eng.device}")
    F = torch.empty((max(n, 1), N_FEAT), dtype=torch.float32, device=Dt.device)
    B = torch.empty(max(n, 1), dtype=torch.float64, device=Dt.device)
    s = np.ascontiguousarray(samples, np.int32)
    _lib.check(eng._L.fjb_router_features(eng._h, Dt.data_ptr(), s.ctypes.data, n, F.data_ptr(),
                                          B.data_ptr()), eng._h)
    return F[:n].cpu().numpy(), B[:n].cpu().numpy()


def training_set(workloads, n_per: int = 20000, seed: int = 0, zero_gap: float = -6.0,
                 label: str = "deposit"):
    """(X, y): features and log10(max|(ab|cd)| x dmax) of sampled computed
    quartets of each workload, the targets from the FP64 HGP tap; with
    label="fp32_error", log10 of the quartet's largest FP32 error into G,
    max|(ab|cd)_FP32 - (ab|cd)_FP64| x dmax (block_err), floored at 10^-14
    of its bound, every computed quartet kept.

    Quartets more than 10^-zero_gap below their Schwarz x density bound are
    left out: they vanish by symmetry (one-centre quartets of odd total
    angular momentum), and what decides their FP32 error is the size of
    their intermediates, which is that of their even siblings, not their
    zero value.  Without them the network treats such quartets like those
    siblings, the conservative side."""
    rng = np.random.default_rng(seed)
    Xs, ys = [], []
    for w in workloads:
        eng = FockEngine(w.basis, tuned=False)
        eng.plan(w.D, w.tau, w.n_mag, export=False)
        s, q = plan_samples(eng, n_per, rng)
        X, b = features(eng, w.D, s)
        keep = b >= w.tau  # computed (not screened) quartets only
        s, X, q = s[keep], X[keep], q[keep]
        if label == "fp32_error":
            y = np.maximum(np.log10(np.maximum(block_err(eng, q), 1e-300)) + X[:, 11], bound_log10(X) - 14.0)
            keep = np.ones(len(y), bool)
        else:
            mx = block_max(eng, q)
            y = np.log10(np.maximum(mx, 1e-300)) + X[:, 11]  # + log10 dmax
            keep = y - bound_log10(X) > zero_gap
        Xs.append(X[keep])
        ys.append(y[keep].astype(np.float32))
        eng.close()
    return np.concatenate(Xs), np.concatenate(ys)


def block_max(eng: FockEngine, quartets: np.ndarray) -> np.ndarray:
    """max |(ab|cd)| of each quartet's block, from the FP64 HGP tap, on the
    device (segment maxima: one pass over the tap's output)."""
    import torch
    q = np.ascontiguousarray(quartets, np.int32)
    n = len(q)
    off = np.zeros(n + 1, np.int64)
    nc = np.array([s.n_cart for s in eng.basis.shells], np.int64)
    off[1:] = np.cumsum(nc[q[:, 0]] * nc[q[:, 1]] * nc[q[:, 2]] * nc[q[:, 3]])
    out = torch.empty(max(int(off[-1]), 1), dtype=torch.float64, device=f"cuda:{eng.device}")
    _lib.check(eng._L.fjb_eri_blocks(eng._h, q.ctypes.data, n, out.data_ptr(), off.ctypes.data), eng._h)
    seg = torch.repeat_interleave(torch.arange(n, device=out.device),
                                  torch.as_tensor(np.diff(off), device=out.device))
    mx = torch.zeros(n, dtype=torch.float64, device=out.device)
    mx.scatter_reduce_(0, seg, out[: int(off[-1])].abs(), reduce="amax", include_self=True)
    return mx.cpu().numpy()


def block_err(eng: FockEngine, quartets: np.ndarray) -> np.ndarray:
    """max |(ab|cd)_FP32 - (ab|cd)_FP64| of each quartet's block: the FP32
    tap (fjb_eri_blocks_fp32, the routed path's FP32 recurrences) against
    the FP64 one, segment maxima on the device."""
    import torch
    q = np.ascontiguousarray(quartets, np.int32)
    n = len(q)
    off = np.zeros(n + 1, np.int64)
    nc = np.array([s.n_cart for s in eng.basis.shells], np.int64)
    off[1:] = np.cumsum(nc[q[:, 0]] * nc[q[:, 1]] * nc[q[:, 2]] * nc[q[:, 3]])
    dev = f"cuda:{eng.device}"
    o64 = torch.empty(max(int(off[-1]), 1), dtype=torch.float64, device=dev)
    o32 = torch.empty_like(o64)
    _lib.check(eng._L.fjb_eri_blocks(eng._h, q.ctypes.data, n, o64.data_ptr(), off.ctypes.data), eng._h)
    _lib.check(eng._L.fjb_eri_blocks_fp32(eng._h, q.ctypes.data, n, o32.data_ptr(), off.ctypes.data), eng._h)
    seg = torch.repeat_interleave(torch.arange(n, device=dev), torch.as_tensor(np.diff(off), device=dev))
    mx = torch.zeros(n, dtype=torch.float64, device=dev)
    m = int(off[-1])
    mx.scatter_reduce_(0, seg, (o32[:m] - o64[:m]).abs(), reduce="amax", include_self=True)
    return mx.cpu().numpy()


def c3_clusters(n: int = 200, lo: int = 8, hi: int = 64, seed: int = 3, first: int = 10_000):
    """Config c3's training systems: n seeded clusters of the c1 shell recipe
    at c1's number density, lo..hi atoms (uniform draw by `seed`), the i-th
    from geometry seed first + i."""
    from . import configs
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=n)
    for i, k in enumerate(sizes):
        yield configs.cluster(int(k), first + i)


def calibrate(mlp: MLP, X, y, quantile: float = 0.999) -> float:
    """The margin: the `quantile` of the residuals y - y_pred (log10 units)."""
    r = y - mlp.predict(X).cpu().numpy()
    return float(np.quantile(r, quantile))


def reach(mlp: MLP, X, margin: float, quantile: float = 0.9999) -> float:
    """The router's reach (decades): the `quantile` of the gaps below the
    Schwarz x density bound the network predicts on X, plus the margin,
    rounded up to a quarter decade and capped at 5.  A quartet whose bound
    is further above the threshold than that would need a larger gap than
    the network gives: the routing pass does not ask it."""
    gap = bound_log10(X) - mlp.predict(X).cpu().numpy()
    r = float(np.quantile(gap, quantile)) + margin
    return float(min(5.0, max(0.0, math.ceil(4.0 * r) / 4.0)))


def install(eng: FockEngine, mlp: MLP, *, threshold: float = 1e-9, margin: float = 0.0,
            reach: float | None = None, min_total_l: int = 0) -> None:
    """Install the network on `eng`: units of classes with total angular
    momentum >= min_total_l whose quartets are within `reach` decades of
    the threshold ask it (fjb_router_reach, fjb_router_classes)."""
    p = np.ascontiguousarray(mlp.params(), np.float32)
    _lib.check(eng._L.fjb_router_set(eng._h, p.ctypes.data,
                                     C.c_float(math.log10(threshold) - margin)), eng._h)
    _lib.check(eng._L.fjb_router_reach(eng._h, 5.0 if reach is None else float(reach)), eng._h)
    _lib.check(eng._L.fjb_router_classes(eng._h, int(min_total_l)), eng._h)


def load_default(device: int = 0) -> tuple[MLP, float, float, int]:
    """The network trained for config c3 (data/router_c3.npz: 7.87 M FP64
    quartets of 200 seeded 8-64-atom clusters, bench.py --path router) with
    its calibrated margin and the reach and class gate measured best on c1
    (0.5 decades, total l >= 7): (network, margin, reach, min_total_l)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "data", "router_c3.npz"))
    return MLP(z["params"], device=device), float(z["margin"]), float(z["reach"]), int(z["min_total_l"])


def uninstall(eng: FockEngine) -> None:
    _lib.check(eng._L.fjb_router_set(eng._h, None, C.c_float(0.0)), eng._h)


def route_stats(eng: FockEngine) -> tuple[int, int]:
    a, b = C.c_int64(), C.c_int64()
    _lib.check(eng._L.fjb_route_stats(eng._h, C.byref(a), C.byref(b)), eng._h)
    return int(a.value), int(b.value)


def validate(eng: FockEngine, D, *, threshold: float = 1e-9, budget: float = 1e-8) -> dict:
    """Build G routed (learned router installed) and in FP64; if max|dG|
    breaks the budget, turn the learned router off (the FP64-side fallback)
    and say so."""
    G64 = eng.build(D, precision=_lib.FJB_FP64)[2].clone()
    Gr = eng.build(D, precision=_lib.FJB_ROUTED, threshold=threshold)[2]
    d = float((Gr - G64).abs().max())
    ok = d <= budget
    if not ok:
        uninstall(eng)
    return {"max_abs_dG": d, "within_budget": ok}
