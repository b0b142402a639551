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
        a_i, b_i = np.triu_indices(na)
        items = np.stack([np.repeat(a_i, nx), np.repeat(b_i, nx), np.tile(np.arange(nx), len(a_i))],
                         axis=1).astype(np.int32)
        out, off = self._blocks(FJB_DF_ERI3, items)
        nc_a = np.array([s.n_cart for s in A.shells])
        nc_x = np.array([s.n_cart for s in X.shells])
        oA, oX = np.asarray(A.offsets), np.asarray(X.offsets)
        sa, sb, sp = nc_a[items[:, 0]], nc_a[items[:, 1]], nc_x[items[:, 2]]
        T = torch.zeros((A.n_ao, A.n_ao, X.n_ao), dtype=torch.float64, device=out.device)
        Tf = T.view(-1)
        dev = out.device
        # one vectorised scatter per block shape (sa, sb, sp)
        for shape in set(zip(sa.tolist(), sb.tolist(), sp.tolist())):
            g = np.nonzero((sa == shape[0]) & (sb == shape[1]) & (sp == shape[2]))[0]
            i, j, k = (x.ravel() for x in np.meshgrid(np.arange(shape[0]), np.arange(shape[1]),
                                                      np.arange(shape[2]), indexing="ij"))
            m = torch.as_tensor(oA[items[g, 0]][:, None] + i[None, :], device=dev)
            n_ = torch.as_tensor(oA[items[g, 1]][:, None] + j[None, :], device=dev)
            p = torch.as_tensor(oX[items[g, 2]][:, None] + k[None, :], device=dev)
            src = torch.as_tensor(off[g][:, None] + np.arange(len(i))[None, :], device=dev)
            vals = out[src]
            nx_ao, n_ao = X.n_ao, A.n_ao
            Tf[(n_ * n_ao + m) * nx_ao + p] = vals
            Tf[(m * n_ao + n_) * nx_ao + p] = vals
        return T

    def factors(self):
        """B = (mn|P) L^{-T} as (n_aux, n_ao, n_ao), FP64, L the metric's
        Cholesky factor.  When the metric is numerically singular (an
        even-tempered aux set on close atoms is nearly linearly dependent
        and the Cholesky breaks down), the factors come from its eigenvectors
        instead: B = Lambda^{-1/2} U^T (P|mn) over the eigenvalues above
        1e-12 of the largest (canonical orthogonalisation), with fewer rows
        than n_aux."""
        import torch
        V = self.metric()
        T = self.eri3().reshape(self.basis.n_ao ** 2, self.aux.n_ao)
        n = self.basis.n_ao
        try:
            L = torch.linalg.cholesky(V)
            B = torch.linalg.solve_triangular(L, T.T, upper=False)  # L^{-1} T^T
        except torch.linalg.LinAlgError:
            w, U = torch.linalg.eigh(V)
            keep = w > 1e-12 * w.max()
            B = (U[:, keep] / torch.sqrt(w[keep])).T @ T.T
        return B.reshape(-1, n, n).contiguous()

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

