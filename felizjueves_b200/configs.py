"""Seeded synthetic inputs for the Fock build: geometries, shells, densities.

The workloads are even-tempered contracted Cartesian shells on random atom
clusters, in the reference's units (Bohr, exponents in Bohr^-2) and its
normalisation convention (coefficients multiply UNNORMALISED primitives;
`primitive_norm` is folded into them here, as `ao/shell.py:84-96` of the
reference describes).

Workloads (sizes are for Cartesian AOs, the reference's convention):

* ``c0``  6 atoms, seed 0, uniform in a 4 A cube, >= 0.9 A apart.  Per atom
  3 s (contraction 3 from 0.15*3^k), 2 p (0.2*3^k), 1 d (0.8): 36 shells,
  90 AO.  D = C C^T, C ~ N(0, 1/n), 12 occupied columns.  tau = 1e-12.
* ``c1``  64 atoms, seed 1, 0.1 atoms/A^3 (cube side 640^(1/3) A), >= 0.95 A
  apart.  Per atom s x3, p x2 (as c0), d x2 (0.8, 2.4), f x1 (1.0): 512
  shells, 1984 AO, 128 occupied columns.  The SCF-like loop perturbs D by
  1e-3 sym(N(0,1)) per build, seeded per iteration.
* ``cluster(n_atoms, seed)``  the c1 shell recipe on n atoms at c1's
  density: used for mid-size parity cases and the uneven molecule batch.

Exponent windows the workload text leaves open (fixed here, once):
s shells take k in {0,1,2}, {2,3,4}, {3,4,5}; p shells {0,1,2}, {3,4,5};
every contraction coefficient is `primitive_norm(l, alpha)`.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .shell import Basis, Shell, primitive_norm

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903

S_WINDOWS = ((0, 1, 2), (2, 3, 4), (3, 4, 5))
P_WINDOWS = ((0, 1, 2), (3, 4, 5))


def _even_tempered(base: float, ratio: float, n: int) -> list[float]:
    return [base * ratio ** k for k in range(n)]


def atom_shells(centre, *, d_exps=(0.8,), f_exps=()) -> list[Shell]:
    """The per-atom shell recipe: 3 contracted s, 2 contracted p, then one
    uncontracted shell per d and f exponent."""
    s_ex = _even_tempered(0.15, 3.0, 6)
    p_ex = _even_tempered(0.2, 3.0, 6)
    out = []
    for w in S_WINDOWS:
        ex = [s_ex[k] for k in w]
        out.append(Shell(0, centre, ex, [primitive_norm(0, e) for e in ex]))
    for w in P_WINDOWS:
        ex = [p_ex[k] for k in w]
        out.append(Shell(1, centre, ex, [primitive_norm(1, e) for e in ex]))
    for a in d_exps:
        out.append(Shell(2, centre, [a], [primitive_norm(2, a)]))
    for a in f_exps:
        out.append(Shell(3, centre, [a], [primitive_norm(3, a)]))
    return out


def sample_geometry(rng: np.random.Generator, n_atoms: int, side_A: float,
                    min_sep_A: float) -> np.ndarray:
    """Sequential rejection sampling: uniform points in [0, side)^3 (A),
    each kept only if it is >= min_sep from every point kept so far.
    Returns Bohr coordinates, shape (n_atoms, 3)."""
    pts: list[np.ndarray] = []
    tries = 0
    while len(pts) < n_atoms:
        x = rng.uniform(0.0, side_A, 3)
        tries += 1
        if tries > 1_000_000:
            raise RuntimeError("rejection sampling did not converge")
        if all(np.linalg.norm(x - y) >= min_sep_A for y in pts):
            pts.append(x)
    return np.asarray(pts) * ANGSTROM_TO_BOHR


def random_density(rng: np.random.Generator, n: int, n_occ: int) -> np.ndarray:
    """D = C C^T with C ~ N(0, 1/n), made bitwise symmetric by (D + D^T)/2
    (the reference refuses an asymmetric density, `ao/density.py:75-100`)."""
    C = rng.normal(0.0, 1.0 / math.sqrt(n), (n, min(n_occ, n)))
    D = C @ C.T
    D = 0.5 * (D + D.T)
    assert np.array_equal(D, D.T)
    return D


@dataclass(frozen=True)
class Workload:
    name: str
    basis: Basis
    D: np.ndarray
    tau: float
    n_mag: int
    coords: np.ndarray
    seed: int
    n_occ: int

    @property
    def n_ao(self) -> int:
        return self.basis.n_ao


def c0() -> Workload:
    rng = np.random.default_rng(0)
    xyz = sample_geometry(rng, 6, 4.0, 0.9)
    shells = [s for c in xyz for s in atom_shells(tuple(map(float, c)))]
    B = Basis(tuple(shells))
    D = random_density(rng, B.n_ao, 12)
    return Workload("c0", B, D, 1e-12, 4, xyz, 0, 12)


C1_DENSITY = 0.1  # atoms per A^3


def cluster(n_atoms: int, seed: int, *, n_occ: int | None = None,
            min_sep_A: float = 0.95, name: str | None = None) -> Workload:
    """`n_atoms` atoms with the c1 shell recipe at c1's number density."""
    rng = np.random.default_rng(seed)
    side = (n_atoms / C1_DENSITY) ** (1.0 / 3.0)
    xyz = sample_geometry(rng, n_atoms, side, min_sep_A)
    shells = [s for c in xyz
              for s in atom_shells(tuple(map(float, c)), d_exps=(0.8, 2.4),
                                   f_exps=(1.0,))]
    B = Basis(tuple(shells))
    if n_occ is None:
        n_occ = 2 * n_atoms
    D = random_density(rng, B.n_ao, n_occ)
    return Workload(name or f"cluster{n_atoms}_s{seed}", B, D, 1e-12, 4, xyz,
                    seed, n_occ)


def c1() -> Workload:
    return cluster(64, 1, n_occ=128, name="c1")


def perturbed_density(D: np.ndarray, iteration: int, *, seed: int = 1,
                      scale: float = 1e-3) -> np.ndarray:
    """D + scale * sym(N(0,1)), seeded by (seed, iteration); bitwise
    symmetric."""
    rng = np.random.default_rng([seed, iteration])
    X = rng.normal(0.0, 1.0, D.shape)
    Dn = D + scale * 0.5 * (X + X.T)
    Dn = 0.5 * (Dn + Dn.T)
    return Dn


def sub_workload(w: Workload, atoms: int) -> Workload:
    """The first `atoms` atoms of `w` (their shells, in order) with the
    matching leading block of its density: a smaller, exactly nested case."""
    per_atom = len(w.basis.shells) // len(w.coords)
    shells = w.basis.shells[: atoms * per_atom]
    B = Basis(tuple(shells))
    D = np.ascontiguousarray(w.D[: B.n_ao, : B.n_ao])
    return Workload(f"{w.name}_{atoms}at", B, D, w.tau, w.n_mag,
                    w.coords[:atoms], w.seed, w.n_occ)


def c4(n_molecules: int = 512) -> list[Workload]:
    """The uneven batch: molecules of 3-40 atoms (uniform size draw from
    seed 4), each a cluster of the c1 shell recipe at c1's density with its
    own seeded geometry and density (n_occ = 2 x atoms).  The first
    `n_molecules` of the 512."""
    rng = np.random.default_rng(4)
    sizes = rng.integers(3, 41, size=512)
    return [cluster(int(n), 4000 + i, name=f"c4_{i}_{int(n)}at")
            for i, n in enumerate(sizes[:n_molecules])]


WORKLOADS = {"c0": c0, "c1": c1}


def by_name(name: str) -> Workload:
    """`c0`, `c1`, or `clusterN` (N atoms of the c1 recipe, seed 5)."""
    if name in WORKLOADS:
        return WORKLOADS[name]()
    if name.startswith("cluster") and name[7:].isdigit():
        return cluster(int(name[7:]), 5)
    raise ValueError(f"unknown workload {name!r}")


# The auxiliary basis recipe (even-tempered s..g, exponents 0.1 * 2.2^k,
# uncontracted, coefficient primitive_norm): per atom s x10, p x7, d x4, f x2,
# g x1 -> 90 Cartesian functions, about 3x the 31 of the c1 shell recipe.
AUX_COUNTS = (10, 7, 4, 2, 1)


def aux_basis(w: Workload) -> Basis:
    shells = []
    for c in w.coords:
        centre = tuple(map(float, c))
        for l, count in enumerate(AUX_COUNTS):
            for k in range(count):
                a = 0.1 * 2.2 ** k
                shells.append(Shell(l, centre, [a], [primitive_norm(l, a)]))
    return Basis(tuple(shells))
