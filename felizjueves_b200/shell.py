"""Contracted Cartesian shells and the basis, in the reference's convention.

Mirrors `ao/shell.py:68-165` of the reference (names, argument meaning and
refusals): coefficients multiply UNNORMALISED Cartesian primitives
x^i y^j z^k exp(-alpha r^2); `primitive_norm(l, alpha)` is the axis-component
normalisation a caller folds in explicitly; the AO order inside a shell is
`cartesians(l)` (i descending, then j descending: xx, xy, xz, yy, yz, zz).
"""

from __future__ import annotations

import math
from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np


def _check_l(l: object) -> int:  # noqa: E741
    if type(l) is not int or l < 0:
        raise ValueError(f"angular momentum {l!r} is not an int >= 0")
    return l


def n_cartesians(l: int) -> int:  # noqa: E741
    _check_l(l)
    return (l + 1) * (l + 2) // 2


def cartesians(l: int) -> tuple[tuple[int, int, int], ...]:  # noqa: E741
    """Every (i, j, k) with i + j + k = l: i descending, then j descending."""
    _check_l(l)
    return tuple((i, j, l - i - j) for i in range(l, -1, -1)
                 for j in range(l - i, -1, -1))


def _dfact_odd(l: int) -> int:  # noqa: E741
    out = 1
    for k in range(1, 2 * l, 2):
        out *= k
    return out


def primitive_norm(l: int, alpha: float) -> float:  # noqa: E741
    """(2 alpha/pi)^(3/4) (4 alpha)^(l/2) / sqrt((2l-1)!!)."""
    _check_l(l)
    if not (isinstance(alpha, (int, float)) and math.isfinite(alpha)
            and alpha > 0):
        raise ValueError(f"exponent {alpha!r} is not a finite float > 0")
    alpha = float(alpha)
    return ((2.0 * alpha / math.pi) ** 0.75 * (4.0 * alpha) ** (l / 2.0)
            / math.sqrt(_dfact_odd(l)))


def _floats(name: str, xs: object) -> tuple[float, ...]:
    if isinstance(xs, (str, bytes)) or not isinstance(xs, (Sequence, np.ndarray)):
        raise ValueError(f"{name} {xs!r} is not a sequence of floats")
    try:
        out = tuple(float(x) for x in xs)
    except (TypeError, ValueError):
        raise ValueError(f"{name} {xs!r} is not a sequence of floats") from None
    if not all(math.isfinite(x) for x in out):
        raise ValueError(f"{name} {xs!r} has a non-finite entry")
    return out


@dataclass(frozen=True)
class Shell:
    l: int  # noqa: E741
    centre: tuple[float, float, float]
    exponents: tuple[float, ...]
    coefficients: tuple[float, ...]

    def __post_init__(self) -> None:
        _check_l(self.l)
        centre = _floats("centre", self.centre)
        if len(centre) != 3:
            raise ValueError(f"centre {self.centre!r} is not three floats")
        ex = _floats("exponents", self.exponents)
        co = _floats("coefficients", self.coefficients)
        if not ex:
            raise ValueError("a shell needs at least one primitive")
        if len(ex) != len(co):
            raise ValueError(f"{len(ex)} exponents but {len(co)} coefficients")
        if not all(a > 0 for a in ex):
            raise ValueError(f"exponents {self.exponents!r} must all be > 0")
        object.__setattr__(self, "centre", centre)
        object.__setattr__(self, "exponents", ex)
        object.__setattr__(self, "coefficients", co)

    @property
    def n_cart(self) -> int:
        return n_cartesians(self.l)

    @property
    def n_prim(self) -> int:
        return len(self.exponents)


@dataclass(frozen=True)
class Basis:
    """Shells in AO order, each shell's first AO index, and the total."""

    shells: tuple[Shell, ...]
    offsets: tuple[int, ...] = field(init=False)
    n_ao: int = field(init=False)

    def __post_init__(self) -> None:
        shells = tuple(self.shells)
        if not all(isinstance(s, Shell) for s in shells):
            raise ValueError("a Basis holds Shells only")
        offsets, n = [], 0
        for s in shells:
            offsets.append(n)
            n += s.n_cart
        object.__setattr__(self, "shells", shells)
        object.__setattr__(self, "offsets", tuple(offsets))
        object.__setattr__(self, "n_ao", n)

    @property
    def n_shells(self) -> int:
        return len(self.shells)

    @property
    def l_max(self) -> int:
        return max((s.l for s in self.shells), default=0)

    def flat(self) -> dict[str, np.ndarray]:
        """The flat arrays the C ABI takes: per shell l, centre (3), first
        primitive index, primitive count, AO offset; and the primitives'
        exponents and coefficients, shell by shell."""
        n = len(self.shells)
        l = np.empty(n, np.int32)
        centre = np.empty((n, 3), np.float64)
        p0 = np.empty(n, np.int32)
        np_ = np.empty(n, np.int32)
        off = np.asarray(self.offsets, np.int32)
        ex, co = [], []
        for i, s in enumerate(self.shells):
            l[i] = s.l
            centre[i] = s.centre
            p0[i] = len(ex)
            np_[i] = len(s.exponents)
            ex.extend(s.exponents)
            co.extend(s.coefficients)
        return {"l": l, "centre": np.ascontiguousarray(centre), "prim0": p0,
                "nprim": np_, "ao_off": off,
                "exps": np.asarray(ex, np.float64),
                "coefs": np.asarray(co, np.float64)}
