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

`jk_streamed(D)` is the same DF-J/K for systems whose (mn|P) does not fit
(c2: 5,760 aux x 1,984^2 AO doubles, 181 GB): the integrals come one aux
block at a time from the library's three-centre Rys kernel (`fjb_df_eri3`),
are contracted at once with D and with D's occupied factors C, and are
discarded; K = Z Z^T with Z = (mi|P) W on the tensor cores (`fjb_df_syrk`),
J from a second pass over the blocks.

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
        self.launches = 0  # the library's kernels launched by eri3_block and syrk
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
        p_i, q_i = np.triu_indices(ns)
        items = np.stack([p_i, q_i], axis=1).astype(np.int32)
        out, off = self._blocks(FJB_DF_METRIC, items)
        nc = np.array([s.n_cart for s in X.shells])
        oX = np.asarray(X.offsets)
        n, dev = X.n_ao, out.device
        V = torch.zeros((n, n), dtype=torch.float64, device=dev)
        sp, sq = nc[p_i], nc[q_i]
        # one vectorised scatter per block shape (np, nq)
        for shape in set(zip(sp.tolist(), sq.tolist())):
            g = np.nonzero((sp == shape[0]) & (sq == shape[1]))[0]
            i, j = (x.ravel() for x in np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), indexing="ij"))
            r = torch.as_tensor(oX[p_i[g]][:, None] + i[None, :], device=dev).reshape(-1)
            c = torch.as_tensor(oX[q_i[g]][:, None] + j[None, :], device=dev).reshape(-1)
            src = torch.as_tensor(off[g][:, None] + np.arange(len(i))[None, :], device=dev).reshape(-1)
            vals = out[src]
            V.index_put_((c, r), vals)
            V.index_put_((r, c), vals)
        return V

    def metric_factor(self, V=None, method: str = "auto"):
        """W with V^{-1} = W W^T on the metric's numerical range: the
        inverse transposed Cholesky factor L^{-T} (n_aux x n_aux), or, when
        the metric is numerically singular (method "auto") or on request
        ("eigh"), U Lambda^{-1/2} over its eigenvalues above 1e-12 of the
        largest (canonical orthogonalisation; fewer columns).  Returns
        (W, L): L is the Cholesky factor, or None for the eigenvector form."""
        import torch
        V = self.metric() if V is None else V
        if method not in ("auto", "cholesky", "eigh"):
            raise ValueError(f"unknown method {method!r}")
        if method != "eigh":
            try:
                L = torch.linalg.cholesky(V)
                I = torch.eye(V.shape[0], dtype=V.dtype, device=V.device)
                return torch.linalg.solve_triangular(L, I, upper=False).T.contiguous(), L
            except torch.linalg.LinAlgError:
                if method == "cholesky":
                    raise
        w, U = torch.linalg.eigh(V)
        keep = w > 1e-12 * w.max()
        return (U[:, keep] / torch.sqrt(w[keep])).contiguous(), None

    def aux_blocks(self, max_functions: int = 384):
        """Consecutive aux shell ranges of at most max_functions functions
        (a shell larger than that is a block of its own): [(s0, s1, p0, p1)]."""
        X = self.aux
        out, s0 = [], 0
        ns = len(X.shells)
        while s0 < ns:
            s1 = s0 + 1
            while s1 < ns and X.offsets[s1] + X.shells[s1].n_cart - X.offsets[s0] <= max_functions:
                s1 += 1
            p1 = X.offsets[s1] if s1 < ns else X.n_ao
            out.append((s0, s1, X.offsets[s0], p1))
            s0 = s1
        return out

    def eri3_block(self, s0: int, s1: int, *, tau: float = 1e-12, out=None, stream=None):
        """(mn|P) for the aux functions of aux shells [s0, s1) by the Rys
        kernel (fjb_df_eri3), n_ao x n_ao x nb ([m][n][P], aux fastest), FP64,
        Schwarz-screened at tau; asynchronous on `stream`."""
        import torch
        X, n = self.aux, self.basis.n_ao
        p0 = X.offsets[s0]
        p1 = X.offsets[s1] if s1 < len(X.shells) else X.n_ao
        if out is None:
            out = torch.empty((n, n, p1 - p0), dtype=torch.float64, device=f"cuda:{self.device}")
        st = stream if stream is not None else torch.cuda.current_stream(out.device)
        nl = C.c_int32()
        _lib.check(self._L.fjb_df_eri3(self._h, int(s0), int(s1), float(tau), out.data_ptr(), C.byref(nl),
                                       C.c_void_p(st.cuda_stream)), self._h)
        self.launches += nl.value
        return out

    def syrk(self, Z, out=None):
        """Z Z^T on the tensor cores (fjb_df_syrk), Z (rows x cols, FP64)."""
        import torch
        Z = Z.contiguous()
        rows, cols = Z.shape
        K = out if out is not None else torch.empty((rows, rows), dtype=torch.float64, device=Z.device)
        st = torch.cuda.current_stream(Z.device)
        self.launches += 2  # the split, the GEMM
        _lib.check(self._L.fjb_df_syrk(self._h, Z.data_ptr(), rows, cols, K.data_ptr(),
                                       C.c_void_p(st.cuda_stream)), self._h)
        return K

    def jk_streamed(self, D, *, tau: float = 1e-12, block: int = 768, mode: str = "bf16x3", factor=None,
                    occ_tol: float = 1e-10, timings: dict | None = None):
        """DF J and K of the symmetric density D (torch, cuda, FP64) without
        holding (mn|P) whole: the integrals are computed one aux block at a
        time (eri3_block), twice.  Pass 1 contracts each block with D
        (d_P = sum_mn (mn|P) D_mn) and with the occupied factors of D
        (Y[m][i][P] = sum_n C_ni (mn|P), D = C_+ C_+^T - C_- C_-^T from its
        eigenvectors over |eigenvalues| above occ_tol of the largest); then
        Z = Y W (W from metric_factor) and K = Z_+ Z_+^T - Z_- Z_-^T
        (mode "bf16x3": fjb_df_syrk on the tensor cores; "fp64": FP64
        GEMMs); c = W W^T d; pass 2 forms J_mn = sum_P (mn|P) c_P.  Memory:
        one block of n_ao^2 block doubles (768 aux functions: 24 GB at
        1,984 AO), Y and Z of n_ao n_occ n_aux each.
        `timings`, if given, receives CUDA-event milliseconds per phase."""
        import torch
        if mode not in ("bf16x3", "fp64"):
            raise ValueError(f"unknown mode {mode!r}")
        dev = D.device
        n, nx = self.basis.n_ao, self.aux.n_ao
        launches0 = self.launches
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        ev[0].record()
        W, L = factor if factor is not None else self.metric_factor()
        ev[5].record()
        w, U = torch.linalg.eigh(D)
        big = w.abs() > occ_tol * w.abs().max()
        Cs = [U[:, big & (w > 0)] * torch.sqrt(w[big & (w > 0)]),
              U[:, big & (w < 0)] * torch.sqrt(-w[big & (w < 0)])]
        ev[1].record()
        blocks = self.aux_blocks(block)
        nbmax = max(p1 - p0 for _, _, p0, p1 in blocks)
        T = torch.empty(n * n * nbmax, dtype=torch.float64, device=dev)
        d = torch.empty(nx, dtype=torch.float64, device=dev)
        Ys = [torch.empty((n, c.shape[1], nx), dtype=torch.float64, device=dev) if c.shape[1] else None
              for c in Cs]
        Dflat = D.reshape(n * n)
        for s0, s1, p0, p1 in blocks:
            Tb = T[: n * n * (p1 - p0)].view(n, n, p1 - p0)
            self.eri3_block(s0, s1, tau=tau, out=Tb)
            d[p0:p1] = Tb.view(n * n, p1 - p0).T @ Dflat
            for c, Y in zip(Cs, Ys):
                if Y is not None:
                    Y[:, :, p0:p1] = torch.matmul(c.T, Tb)
        ev[2].record()
        K = torch.zeros((n, n), dtype=torch.float64, device=dev)
        for idx, sign in ((0, 1.0), (1, -1.0)):
            Y, Ys[idx] = Ys[idx], None
            if Y is None:
                continue
            o = Cs[idx].shape[1]
            if L is not None:  # Z = Y L^{-T}: the triangular solve, half the GEMM's work
                Z = torch.linalg.solve_triangular(L.T, Y.view(n * o, nx), upper=True, left=False)
            else:
                Z = Y.view(n * o, nx) @ W
            del Y
            Zm = Z.contiguous().view(n, -1)  # the solve may return it column-major
            Kp = self.syrk(Zm) if mode == "bf16x3" else Zm @ Zm.T
            K += sign * Kp
            del Z, Zm, Kp
        ev[3].record()
        cvec = W @ (W.T @ d)
        J = torch.zeros(n * n, dtype=torch.float64, device=dev)
        for s0, s1, p0, p1 in blocks:
            Tb = T[: n * n * (p1 - p0)].view(n, n, p1 - p0)
            self.eri3_block(s0, s1, tau=tau, out=Tb)
            J += Tb.view(n * n, p1 - p0) @ cvec[p0:p1]
        ev[4].record()
        if timings is not None:
            torch.cuda.synchronize(dev)
            timings.update({"factor_ms": ev[0].elapsed_time(ev[5]), "occupied_ms": ev[5].elapsed_time(ev[1]),
                            "pass1_ms": ev[1].elapsed_time(ev[2]),
                            "k_ms": ev[2].elapsed_time(ev[3]), "pass2_ms": ev[3].elapsed_time(ev[4]),
                            "blocks": len(blocks), "n_occ": [int(c.shape[1]) for c in Cs],
                            "fjb_launches": self.launches - launches0,
                            "aux_kept": int(W.shape[1])})
        return J.view(n, n), 0.5 * (K + K.T)

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

