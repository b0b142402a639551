"""ctypes front end of the CPU oracle (oracle.c). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (felizjueves_b200) never does.  `build()` compiles
oracle.c with the Makefile beside it into oracle/_build/liboracle.so.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


class _Basis(C.Structure):
    _fields_ = [("n_sh", C.c_int), ("l", C.c_void_p), ("centre", C.c_void_p),
                ("prim0", C.c_void_p), ("nprim", C.c_void_p), ("exps", C.c_void_p),
                ("coefs", C.c_void_p), ("ao_off", C.c_void_p), ("n_ao", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.or_boys.restype = C.c_double
        L.or_boys.argtypes = [C.c_int, C.c_double]
        L.or_eri_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_void_p]
        L.or_jk_ordered.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int]
        L.or_jk_unique.argtypes = L.or_jk_ordered.argtypes
        L.or_fock_quartets.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p]
        _lib = L
    return _lib


class OracleBasis:
    """Keeps the flat arrays alive for the C struct that points at them."""

    def __init__(self, l, centre, prim0, nprim, exps, coefs):
        self.l = np.ascontiguousarray(l, np.int32)
        self.centre = np.ascontiguousarray(centre, np.float64).reshape(-1, 3)
        self.prim0 = np.ascontiguousarray(prim0, np.int32)
        self.nprim = np.ascontiguousarray(nprim, np.int32)
        self.exps = np.ascontiguousarray(exps, np.float64)
        self.coefs = np.ascontiguousarray(coefs, np.float64)
        nc = (self.l + 1) * (self.l + 2) // 2
        self.ao_off = np.ascontiguousarray(np.concatenate([[0], np.cumsum(nc)[:-1]]),
                                           np.int32)
        self.n_ao = int(nc.sum())
        self.ncart = nc
        self.s = _Basis(len(self.l), self.l.ctypes.data, self.centre.ctypes.data,
                        self.prim0.ctypes.data, self.nprim.ctypes.data,
                        self.exps.ctypes.data, self.coefs.ctypes.data,
                        self.ao_off.ctypes.data, self.n_ao)

    @classmethod
    def of(cls, basis):
        """From a felizjueves_b200.shell.Basis."""
        f = basis.flat()
        return cls(f["l"], f["centre"], f["prim0"], f["nprim"], f["exps"], f["coefs"])

    @classmethod
    def from_npz(cls, z):
        return cls(z["l"], z["centre"], z["prim0"], z["nprim"], z["exps"], z["coefs"])


def boys(m: int, T: float) -> float:
    return lib().or_boys(int(m), float(T))


def eri_block(ob: OracleBasis, a, b, c, d, want_scale=False):
    n = [int(ob.ncart[x]) for x in (a, b, c, d)]
    out = np.zeros(n[0] * n[1] * n[2] * n[3])
    sc = np.zeros_like(out) if want_scale else None
    rc = lib().or_eri_block(C.byref(ob.s), a, b, c, d, out.ctypes.data,
                            sc.ctypes.data if sc is not None else None)
    if rc:
        raise ValueError(f"oracle eri_block refused: {rc}")
    return (out, sc) if want_scale else out


def jk(ob: OracleBasis, D, *, ordered=False, threads=0):
    """(J, K) of the density D by the every-ordered-quartet sweep
    (`ordered=True`) or by one quartet per 8-fold orbit."""
    D = np.ascontiguousarray(D, np.float64)
    n = ob.n_ao
    assert D.shape == (n, n)
    J = np.zeros((n, n))
    K = np.zeros((n, n))
    fn = lib().or_jk_ordered if ordered else lib().or_jk_unique
    rc = fn(C.byref(ob.s), D.ctypes.data, J.ctypes.data, K.ctypes.data, int(threads))
    if rc:
        raise ValueError(f"oracle jk refused: {rc}")
    return J, K


def fock_quartets(ob: OracleBasis, D, quartets, degs, kept=None, threads=0):
    """The reference's per-quartet work of the fused build (ERI block + the
    six-block digest) on a list of unique quartets, timed per quartet on
    `threads` OpenMP threads.  `kept`: per quartet a (bra, ket) pair of
    kept-primitive index lists (the plan's pruned pairs), or None for every
    primitive.  Returns (J, K, seconds per quartet); J, K unclosed."""
    D = np.ascontiguousarray(D, np.float64)
    q = np.ascontiguousarray(quartets, np.int32).reshape(-1, 4)
    n = len(q)
    dg = np.ascontiguousarray(degs, np.float64)
    assert dg.shape == (n,)
    koff = kidx = None
    if kept is not None:
        lists = [lst for pair in kept for lst in pair]
        assert len(lists) == 2 * n
        koff = np.ascontiguousarray(np.concatenate([[0], np.cumsum([len(x) for x in lists])]), np.int32)
        kidx = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in lists])
                                    if n else np.zeros(1, np.int32), np.int32)
    J = np.zeros((ob.n_ao, ob.n_ao))
    K = np.zeros_like(J)
    sec = np.zeros(max(n, 1))
    rc = lib().or_fock_quartets(C.byref(ob.s), D.ctypes.data, n, q.ctypes.data, dg.ctypes.data,
                                koff.ctypes.data if koff is not None else None,
                                kidx.ctypes.data if kidx is not None else None,
                                J.ctypes.data, K.ctypes.data, int(threads), sec.ctypes.data)
    if rc:
        raise ValueError(f"oracle fock_quartets refused: {rc}")
    return J, K, sec[:n]
