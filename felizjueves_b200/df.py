"""Density fitting: the (P|Q) metric and (mn|P) three-centre integrals on the
GPU, and DF-J/K built from them.

Mirrors `eri/density_fit/metric.py:228 metric_matrix` and
`eri/density_fit/eri3.py:226 eri3_tensor` of the reference (layouts: (P|Q)
rows and columns in aux-basis AO order; (mn|P) as [m][n][P], aux fastest,
mirrored in (m, n)).  The integrals come from libfjb's HGP kernels
(`fjb_df_blocks`).  The reference computes no DF-J/K (density_fit/
__init__.py:8-9); the contraction here is the standard one, with the metric's
Cholesky factor L (V = L L^T):

    B = (mn|P) L^{-T}                          (n_ao^2 x n_aux)
    J_mn = sum_P B_mn,P (sum_ls B_ls,P D_ls)
    K_mn = sum_P sum_ls B_ml,P D_ls B_sn,P

`jk(D, mode="bf16x3")` runs the contractions through the library's own
kernels (`fjb_df_jk`, csrc/df_mm.cu): J by two FP64 passes over B, K by two
GEMMs on the tensor cores (tcgen05, accumulators in tensor memory) as split
products -- each FP32 operand the sum of three BF16 terms (hi + mid + lo),
the six products whose orders sum to at most 2 accumulated in FP32, which
keeps the FP32 operand's precision to about 2^-24.  `mode="fp64"` is the
FP64 check path (device FP64 GEMMs through torch).  The Cholesky and the
triangular solve are FP64.  Errors of both against the exact (4-centre) J,
K are reported by the tests.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .shell import Basis

FJB_DF_METRIC = 0
FJB_DF_ERI3 = 1


def _basis_t(basis: Basis):
    f = basis.flat()
    bt = _lib.Basis_t(len(basis.shells), f["l"].ctypes.data, f["centre"].ctypes.data,
                      f["prim0"].ctypes.data, f["nprim"].ctypes.data,
                      f["exps"].ctypes.data, f["coefs"].ctypes.data)
    return bt, f


class DFEngine:
    """The AO basis and an auxiliary basis on one GPU."""

    def __init__(self, basis: Basis, aux: Basis, device: int = 0):
        self.basis, self.aux, self.device = basis, aux, int(device)
        self._L = _lib.load()
        a, self._fa = _basis_t(basis)
        x, self._fx = _basis_t(aux)
        h = C.c_void_p()
        _lib.check(self._L.fjb_create_df(C.byref(h), C.byref(a), C.byref(x), self.device))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.fjb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _blocks(self, kind: int, items: np.ndarray):
        import torch
        items = np.ascontiguousarray(items, np.int32)
        n = len(items)
        off = np.zeros(n + 1, np.int64)
        # sizes first, to allocate the output once
        if kind == FJB_DF_METRIC:
            sz = [self.aux.shells[p].n_cart * self.aux.shells[q].n_cart for p, q in items]
        else:
            sz = [self.basis.shells[a].n_cart * self.basis.shells[b].n_cart *
                  self.aux.shells[p].n_cart for a, b, p in items]
        out = torch.empty(max(int(np.sum(sz)), 1), dtype=torch.float64,
                          device=f"cuda:{self.device}")
        _lib.check(self._L.fjb_df_blocks(self._h, kind, items.ctypes.data, n, out.data_ptr(),
                                         off.ctypes.data), self._h)
        return out, off

    def metric(self):
        """(P|Q), n_aux x n_aux, FP64 on the device, exactly symmetric."""
        import torch
        X = self.aux
        ns = len(X.shells)
        items = np.array([(p, q) for p in range(ns) for q in range(p, ns)], np.int32)
        out, off = self._blocks(FJB_DF_METRIC, items)
        rows, cols = [], []
        for (p, q) in items:
            np_, nq = X.shells[p].n_cart, X.shells[q].n_cart
            r = X.offsets[p] + np.repeat(np.arange(np_), nq)
            c = X.offsets[q] + np.tile(np.arange(nq), np_)
            rows.append(r)
            cols.append(c)
        rows, cols = np.concatenate(rows), np.concatenate(cols)
        n = X.n_ao
        V = torch.zeros((n, n), dtype=torch.float64, device=out.device)
        ri = torch.as_tensor(rows, device=out.device)
        ci = torch.as_tensor(cols, device=out.device)
        vals = out[: len(rows)]
        V.index_put_((ci, ri), vals)
        V.index_put_((ri, ci), vals)
        return V

    def eri3(self):
        """(mn|P), n_ao x n_ao x n_aux ([m][n][P], aux fastest), FP64."""
        import torch
        A, X = self.basis, self.aux
        na, nx = len(A.shells), len(X.shells)
        items = np.array([(a, b, p) for a in range(na) for b in range(a, na) for p in range(nx)],
                         np.int32)
        out, off = self._blocks(FJB_DF_ERI3, items)
        m_idx, n_idx, p_idx = [], [], []
        for (a, b, p) in items:
            sa, sb, sp = A.shells[a].n_cart, A.shells[b].n_cart, X.shells[p].n_cart
            i, j, k = np.meshgrid(np.arange(sa), np.arange(sb), np.arange(sp), indexing="ij")
            m_idx.append(A.offsets[a] + i.ravel())
            n_idx.append(A.offsets[b] + j.ravel())
            p_idx.append(X.offsets[p] + k.ravel())
        mi = torch.as_tensor(np.concatenate(m_idx), device=out.device)
        ni = torch.as_tensor(np.concatenate(n_idx), device=out.device)
        pi = torch.as_tensor(np.concatenate(p_idx), device=out.device)
        T = torch.zeros((A.n_ao, A.n_ao, X.n_ao), dtype=torch.float64, device=out.device)
        vals = out[: len(mi)]
        T.index_put_((ni, mi, pi), vals)
        T.index_put_((mi, ni, pi), vals)
        return T

    def factors(self):
        """B = (mn|P) L^{-T} as (n_aux, n_ao, n_ao), FP64."""
        import torch
        V = self.metric()
        L = torch.linalg.cholesky(V)
        T = self.eri3().reshape(self.basis.n_ao ** 2, self.aux.n_ao)
        B = torch.linalg.solve_triangular(L, T.T, upper=False)  # L^{-1} T^T
        n = self.basis.n_ao
        return B.reshape(self.aux.n_ao, n, n)

    def jk(self, D, mode: str = "fp64", B=None):
        """(J, K) of the density D (torch, cuda, FP64) by density fitting."""
        import torch
        if B is None:
            B = self.factors()
        nx, n, _ = B.shape
        if mode == "fp64":
            gamma = B.reshape(nx, n * n) @ D.reshape(n * n)
            J = (B.reshape(nx, n * n).T @ gamma).reshape(n, n)
            X = torch.matmul(B, D)                                  # (nx, n, n)
            K = torch.matmul(X.permute(1, 0, 2).reshape(n, nx * n),
                             B.permute(0, 2, 1).reshape(nx * n, n))
            return J, K
        if mode == "bf16x3":
            # the library's kernels (fjb_df_jk): J in FP64, K on the tensor
            # cores as split-BF16 products accumulated in FP32
            Bc = B.contiguous()
            Dc = D.contiguous()
            J = torch.empty((n, n), dtype=torch.float64, device=Bc.device)
            K = torch.empty_like(J)
            st = torch.cuda.current_stream(Bc.device)
            _lib.check(self._L.fjb_df_jk(self._h, Bc.data_ptr(), nx, n, Dc.data_ptr(), J.data_ptr(),
                                         K.data_ptr(), C.c_void_p(st.cuda_stream)), self._h)
            return J, K
        raise ValueError(f"unknown mode {mode!r}")

