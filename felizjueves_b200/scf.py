"""Closed-shell SCF around the G build: the caller of the hot path.

    rhf(basis, nuclei, ...) -> SCFResult

The loop a user of the reference runs around `fock_two_electron`: the
one-electron matrices S and H = T + V (`fjb_one_electron`), the symmetric
orthogonaliser X = S^{-1/2}, the core-Hamiltonian guess, then per iteration
F = H + G(D), the energy E = 1/2 tr D (H + F) + E_nuc, Pulay DIIS on the
commutator X^T (F D S - S D F) X, and D = 2 C_occ C_occ^T from the
generalised eigenproblem F C = S C e (torch.linalg.eigh on the device).

G(D) comes from the sm_100a Fock build.  With `incremental=True` (the
default) an iteration builds G(D_k) = G(D_g) + G(D_k - D_g) from the last
built density D_g: the plan and the six-block screen run on the difference
density, so a quartet drops out once |dD| G_ab G_cd falls below tau (in
large systems, late in the loop; in a small molecule |dD| ~ 1e-9 keeps
nearly every quartet above tau = 1e-12); every `rebuild_every`-th
iteration, and the first, builds G(D) in full so screening errors of the
differences do not accumulate.  D is kept exactly symmetric ((D + D^T) / 2), which the plan
requires.

The reference has no SCF driver; its J/K/G drivers take the density as
given.  `builders` injects the one-electron and G evaluators (the reference's
own style, eri/fock/fock.py:126-176 take `eri=`); the default is the GPU
engine, and the loop's linear algebra runs on the builders' device.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .fock import FockEngine, _checked_nuclei
from .shell import Basis


@dataclass
class SCFResult:
    energy: float              # total: electronic + nuclear repulsion
    e_nuc: float
    mo_energy: np.ndarray
    mo_coeff: np.ndarray
    D: np.ndarray              # the converged total density
    iterations: int
    converged: bool
    history: list = field(default_factory=list)  # per iteration: (energy, max|dD|, "full"|"delta")


def nuclear_repulsion(nuclei) -> float:
    nuc = _checked_nuclei(nuclei)
    e = 0.0
    for i in range(len(nuc)):
        for j in range(i):
            zi, ci = nuc[i]
            zj, cj = nuc[j]
            r = math.dist(ci, cj)
            if r == 0.0:
                raise ValueError(f"nuclei {j} and {i} coincide")
            e += zi * zj / r
    return e


class GpuBuilders:
    """The one-electron matrices and G(D) from the sm_100a kernels."""

    def __init__(self, basis: Basis, *, device: int = 0, tau: float = 1e-12, n_mag: int = 4,
                 precision: int = _lib.FJB_FP64, threshold: float = 0.0):
        import torch
        self.eng = FockEngine(basis, device)
        self.device = torch.device(f"cuda:{device}")
        self.tau, self.n_mag = tau, n_mag
        self.precision, self.threshold = precision, threshold
        self.computed = []  # quartets the six-block screen let through, per G build

    def one_electron(self, nuclei):
        S, _, _, H = self.eng.one_electron(nuclei, want=("S", "H"))
        return S, H

    def g(self, D):
        self.eng.plan(D.cpu().numpy(), self.tau, self.n_mag, export=False)
        G = self.eng.build(D, precision=self.precision, threshold=self.threshold)[2]
        self.computed.append(sum(st["computed"] for st in self.eng.launch_stats()))
        return G


def rhf(basis: Basis, nuclei, *, n_elec: int | None = None, tau: float = 1e-12, n_mag: int = 4,
        precision: int = _lib.FJB_FP64, threshold: float = 0.0, incremental: bool = True,
        rebuild_every: int = 8, max_iter: int = 100, e_tol: float = 1e-10, d_tol: float = 1e-8,
        diis_size: int = 8, device: int = 0, builders=None) -> SCFResult:
    """Closed-shell SCF of `basis` in the field of `nuclei` [(Z, (x, y, z))]
    (Bohr), n_elec electrons (default: the neutral molecule).  Converged when
    the energy changes by < e_tol and the density by < d_tol (max-abs)."""
    import torch
    nuc = _checked_nuclei(nuclei)
    if n_elec is None:
        n_elec = int(round(sum(z for z, _ in nuc)))
    if n_elec <= 0 or n_elec % 2:
        raise ValueError(f"n_elec = {n_elec}: a closed shell needs an even count > 0")
    n_occ = n_elec // 2
    if n_occ > basis.n_ao:
        raise ValueError(f"{n_occ} occupied orbitals but {basis.n_ao} AOs")
    if rebuild_every < 1:
        raise ValueError("rebuild_every must be >= 1")
    b = builders if builders is not None else GpuBuilders(basis, device=device, tau=tau, n_mag=n_mag,
                                                          precision=precision, threshold=threshold)
    e_nuc = nuclear_repulsion(nuc)
    S, H = b.one_electron(nuc)
    s, U = torch.linalg.eigh(S)
    if float(s.min()) <= 1e-10 * float(s.max()):
        raise ValueError(f"the overlap is near-singular (smallest eigenvalue {float(s.min()):.3e})")
    X = (U * s.rsqrt()) @ U.T

    def solve(F):
        e, Cp = torch.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        Co = C[:, :n_occ]
        D = 2.0 * (Co @ Co.T)
        return e, C, 0.5 * (D + D.T)

    e, C, D = solve(H)
    G = Dg = None
    E_prev = None
    errs, focks = [], []
    hist = []
    converged = False
    it = 0
    for it in range(1, max_iter + 1):
        full = G is None or not incremental or (it - 1) % rebuild_every == 0
        if full:
            G = b.g(D)
        else:
            G = G + b.g(D - Dg)
        Dg = D
        F = H + G
        E = 0.5 * float((D * (H + F)).sum()) + e_nuc
        # DIIS on the orthogonalised commutator
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        errs.append(err)
        focks.append(F)
        if len(errs) > diis_size:
            errs.pop(0)
            focks.pop(0)
        m = len(errs)
        if m > 1:
            B = torch.empty((m + 1, m + 1), dtype=F.dtype, device=F.device)
            for i in range(m):
                for j in range(i, m):
                    B[i, j] = B[j, i] = (errs[i] * errs[j]).sum()
            B[m, :m] = B[:m, m] = -1.0
            B[m, m] = 0.0
            rhs = torch.zeros(m + 1, dtype=F.dtype, device=F.device)
            rhs[m] = -1.0
            c = torch.linalg.lstsq(B.cpu(), rhs.cpu().unsqueeze(1)).solution.squeeze(1).to(F.device)
            Fx = sum(c[i] * focks[i] for i in range(m))
            Fx = 0.5 * (Fx + Fx.T)
        else:
            Fx = F
        e, C, Dn = solve(Fx)
        dmax = float((Dn - D).abs().max())
        hist.append((E, dmax, "full" if full else "delta"))
        done = E_prev is not None and abs(E - E_prev) < e_tol and dmax < d_tol
        E_prev = E
        D = Dn
        if done:
            converged = True
            # orbitals of the converged Fock matrix itself (no extrapolation)
            e, C, _ = solve(F)
            break
    return SCFResult(energy=E_prev, e_nuc=e_nuc, mo_energy=e.cpu().numpy(), mo_coeff=C.cpu().numpy(),
                     D=D.cpu().numpy(), iterations=it, converged=converged, history=hist)
