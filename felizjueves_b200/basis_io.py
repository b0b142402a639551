"""Basis sets from Basis Set Exchange JSON, mapped onto this package's shells.

    parse(doc) / load(path) -> BasisSet          ao/bse.py:143-170 parse, load
    from_bse(basis_set, atoms, reduce=False) -> Basis
                                                 test/oracle/basis.py from_bse

Reading (`parse`) keeps the document's numbers as they are: a fused shell
(`"angular_momentum": [0, 1]`, Pople's SP) becomes one `Contraction` per
angular momentum with its own coefficient row; a general contraction (one
angular momentum, several rows, as in cc-pVDZ) stays one `Contraction` with
several rows, zero entries kept; `function_type` is recorded only (every AO
here is Cartesian, so a `gto_spherical` d is six functions).

Mapping (`from_bse`) gives the shells libcint integrates for the same file
with `cart=True`, in libcint's AO order:
  * order: an element's contractions by angular momentum, file order within
    one (`libcint_order`);
  * coefficients: each file coefficient times the radial normaliser
    gto_norm(l, a) = 1/sqrt(int r^(2l+2) e^(-2 a r^2) dr), the row scaled to
    unit radial norm, times libcint's common factor (1/sqrt(4 pi) for s,
    sqrt(3/(4 pi)) for p, 1 from d up) -- the convention of this package's
    `Shell`, whose coefficients multiply unnormalised primitives;
  * `reduce=True` takes the free-primitive-reduced form the correlation-
    consistent sets have in PySCF's library: a primitive that stands alone
    (one exponent, coefficient 1) is removed from the contracted functions of
    its angular momentum and kept as its own function after them.
"""

from __future__ import annotations

import json
import math
from collections.abc import Mapping, Sequence
from dataclasses import dataclass
from pathlib import Path
from types import MappingProxyType

from .shell import Basis, Shell

FUNCTION_TYPES = frozenset({"gto", "gto_spherical", "gto_cartesian"})


@dataclass(frozen=True)
class Contraction:
    l: int  # noqa: E741
    exponents: tuple[float, ...]
    coefficients: tuple[tuple[float, ...], ...]  # one row per contracted function
    function_type: str = "gto"


@dataclass(frozen=True)
class BasisSet:
    name: str
    elements: Mapping[int, tuple[Contraction, ...]]

    def contractions(self, z: int) -> tuple[Contraction, ...]:
        try:
            return self.elements[int(z)]
        except KeyError:
            raise ValueError(f"{self.name} has no element Z = {z}") from None


def _numbers(where: str, xs) -> tuple[float, ...]:
    if isinstance(xs, (str, bytes)) or not isinstance(xs, Sequence):
        raise ValueError(f"{where}: {xs!r} is not a list of numbers")
    try:
        out = tuple(float(x) for x in xs)
    except (TypeError, ValueError):
        raise ValueError(f"{where}: {xs!r} holds a non-number") from None
    if not all(math.isfinite(x) for x in out):
        raise ValueError(f"{where}: a non-finite number")
    return out


def _shell(where: str, raw) -> tuple[Contraction, ...]:
    if not isinstance(raw, Mapping):
        raise ValueError(f"{where}: not an object")
    ft = raw.get("function_type")
    if ft not in FUNCTION_TYPES:
        raise ValueError(f"{where}: function_type {ft!r} is not one of {sorted(FUNCTION_TYPES)}")
    ams = raw.get("angular_momentum")
    if not isinstance(ams, Sequence) or not ams or not all(isinstance(l, int) and l >= 0 for l in ams):
        raise ValueError(f"{where}: angular_momentum {ams!r} is not a list of ints >= 0")
    ex = _numbers(f"{where} exponents", raw.get("exponents"))
    if not ex or not all(a > 0 for a in ex):
        raise ValueError(f"{where}: exponents must be > 0")
    rows = raw.get("coefficients")
    if not isinstance(rows, Sequence) or not rows:
        raise ValueError(f"{where}: no coefficients")
    rows = tuple(_numbers(f"{where} coefficients", r) for r in rows)
    if any(len(r) != len(ex) for r in rows):
        raise ValueError(f"{where}: a coefficient row does not match the {len(ex)} exponents")
    if len(ams) == 1:
        return (Contraction(ams[0], ex, rows, ft),)
    if len(rows) != len(ams):
        raise ValueError(f"{where}: a fused shell needs one coefficient row per angular momentum")
    return tuple(Contraction(l, ex, (r,), ft) for l, r in zip(ams, rows))


def parse(doc) -> BasisSet:
    """A BSE JSON document (molssi_bse_schema) as a BasisSet."""
    if not isinstance(doc, Mapping) or not isinstance(doc.get("elements"), Mapping):
        raise ValueError("not a Basis Set Exchange document: no 'elements'")
    name = str(doc.get("name", "?"))
    els = {}
    for z, el in doc["elements"].items():
        shells = el.get("electron_shells") if isinstance(el, Mapping) else None
        if not isinstance(shells, Sequence):
            raise ValueError(f"{name} Z = {z}: no electron_shells")
        cs = []
        for k, sh in enumerate(shells):
            cs.extend(_shell(f"{name} Z = {z} shell {k}", sh))
        els[int(z)] = tuple(cs)
    return BasisSet(name, MappingProxyType(els))


def load(path: str | Path) -> BasisSet:
    with open(path) as fh:
        return parse(json.load(fh))


def canonical(name: str) -> str:
    """The matching key of a set's name: case ignored, '-', '_' and spaces
    dropped (ao/bse.py:171)."""
    return "".join(ch for ch in name.lower() if ch not in "-_ ")


def _gaussian_int(n: int, a: float) -> float:
    """int_0^inf r^n e^(-a r^2) dr."""
    return math.gamma((n + 1) / 2.0) / (2.0 * a ** ((n + 1) / 2.0))


def gto_norm(l: int, a: float) -> float:  # noqa: E741
    return 1.0 / math.sqrt(_gaussian_int(2 * l + 2, 2.0 * a))


def common_factor(l: int) -> float:  # noqa: E741
    if l == 0:
        return 1.0 / math.sqrt(4.0 * math.pi)
    if l == 1:
        return math.sqrt(3.0 / (4.0 * math.pi))
    return 1.0


def libcint_order(cs: Sequence[Contraction]) -> tuple[Contraction, ...]:
    return tuple(sorted(cs, key=lambda c: c.l))


def free_primitive_reduced(cs: Sequence[Contraction]) -> tuple[Contraction, ...]:
    """Per angular momentum (ascending): every contracted function with its
    zero entries and its components on a free exponent dropped, in file
    order, then every free primitive alone."""
    out = []
    for l in sorted({c.l for c in cs}):  # noqa: E741
        funcs = []
        for c in cs:
            if c.l == l:
                for row in c.coefficients:
                    funcs.append([(a, x) for a, x in zip(c.exponents, row) if x != 0.0])
        free = {f[0][0] for f in funcs if len(f) == 1 and f[0][1] == 1.0}
        alone = []
        for f in funcs:
            if len(f) == 1 and f[0][1] == 1.0:
                alone.append(f[0][0])
                continue
            keep = [(a, x) for a, x in f if a not in free]
            out.append(Contraction(l, tuple(a for a, _ in keep), (tuple(x for _, x in keep),)))
        out.extend(Contraction(l, (a,), ((1.0,),)) for a in alone)
    return tuple(out)


def mapped_coefficients(c: Contraction) -> tuple[tuple[float, ...], ...]:
    """This package's coefficients for each contracted function of `c`."""
    l = c.l  # noqa: E741
    g = [gto_norm(l, a) for a in c.exponents]
    out = []
    for row in c.coefficients:
        w = [x * gp for x, gp in zip(row, g)]
        s = sum(wp * wq * _gaussian_int(2 * l + 2, ap + aq)
                for wp, ap in zip(w, c.exponents) for wq, aq in zip(w, c.exponents))
        if not s > 0.0:
            raise ValueError(f"a contraction of l = {l} has zero norm")
        k = common_factor(l) / math.sqrt(s)
        out.append(tuple(wp * k for wp in w))
    return tuple(out)


def from_bse(basis_set: BasisSet, atoms, *, reduce: bool = False) -> Basis:
    """Shells for `atoms` [(Z, (x, y, z)) in Bohr] in `basis_set`, libcint's
    AO order, one Shell per contracted function."""
    shells = []
    for z, centre in atoms:
        cs = basis_set.contractions(int(round(float(z))))
        for c in (free_primitive_reduced(cs) if reduce else libcint_order(cs)):
            shells.extend(Shell(c.l, tuple(float(x) for x in centre), c.exponents, row)
                          for row in mapped_coefficients(c))
    return Basis(tuple(shells))
