"""Uneven batched builds: many molecules of different sizes.

Each molecule keeps its own handle, plan and device buffers (D, J, K, G).
Two ways to build them together:

* `merged` (the batched build, fjb_batch_*): every molecule's work units of
  a class in ONE class-sorted queue, so the whole batch is one launch per
  angular-momentum class (55 for l <= 3), each a persistent grid pulling
  units from the queue and finding the unit's molecule (its density, its
  J', K') through the unit's launch; one launch makes every molecule's
  density blocks and one closes every molecule's J, K, G.  `capture_merged`
  records it as one CUDA graph.
* `capture`: every molecule's own build (its class launches, FP64 or routed
  with the learned router) recorded back to back into one CUDA graph; each
  molecule's device time is read back after a replay (`device_ms`).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .fock import FockEngine


class BatchBuilder:
    def __init__(self, workloads, device: int = 0):
        import torch
        self.workloads = list(workloads)
        self.device = int(device)
        dev = f"cuda:{self.device}"
        self.engines, self.D, self.out = [], [], []
        for w in self.workloads:
            eng = FockEngine(w.basis, device=self.device)
            eng.plan(w.D, w.tau, w.n_mag, export=False)
            self.engines.append(eng)
            D = torch.tensor(w.D, device=dev)
            self.D.append(D)
            self.out.append(tuple(torch.empty_like(D) for _ in range(3)))
        self.graphs = {}
        self._batch = None

    def build_loop(self, precision: int = _lib.FJB_FP64, threshold: float = 0.0):
        """Every molecule's build, one after another, each its own calls."""
        for eng, D, (J, K, G) in zip(self.engines, self.D, self.out):
            eng.build(D, J=J, K=K, G=G, precision=precision, threshold=threshold)

    def capture(self, key, precision: int = _lib.FJB_FP64, threshold: float = 0.0) -> None:
        """Record the whole batch's builds as one CUDA graph under `key`."""
        import torch
        self.build_loop(precision, threshold)  # warm: first-use staging happens outside the capture
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.build_loop(precision, threshold)
        self.graphs[key] = g

    def replay(self, key) -> None:
        self.graphs[key].replay()

    def device_ms(self) -> np.ndarray:
        """Per molecule: the device time of its last build's class kernels."""
        return np.array([eng.last_build_stats()[0] for eng in self.engines])

    def G(self):
        return [o[2] for o in self.out]

    # -- the batched build (one launch per class for the whole batch) -----
    def _merged(self):
        if self._batch is None:
            L = _lib.load()
            n = len(self.engines)
            hs = (C.c_void_p * n)(*[e._h.value for e in self.engines])
            b = C.c_void_p()
            rc = L.fjb_batch_create(C.byref(b), C.cast(hs, C.c_void_p), n)
            if rc:
                raise RuntimeError(f"fjb_batch_create: {L.fjb_batch_last_error(None).decode()}")
            ptrs = [(C.c_void_p * n)(*[t.data_ptr() for t in col])
                    for col in (self.D, [o[0] for o in self.out], [o[1] for o in self.out],
                                [o[2] for o in self.out])]
            rc = L.fjb_batch_set_densities(b, *[C.cast(p, C.c_void_p) for p in ptrs])
            if rc:
                raise RuntimeError(f"fjb_batch_set_densities: {L.fjb_batch_last_error(b).decode()}")
            self._batch = b
        return self._batch

    def build_merged(self, precision: int = _lib.FJB_FP64, threshold: float = 0.0) -> None:
        """The batch in one launch per class (stream-ordered)."""
        import torch
        L = _lib.load()
        b = self._merged()
        st = torch.cuda.current_stream(self.device)
        rc = L.fjb_batch_build(b, int(precision), float(threshold), C.c_void_p(st.cuda_stream))
        if rc:
            raise RuntimeError(f"fjb_batch_build: {L.fjb_batch_last_error(b).decode()}")

    def capture_merged(self, key, precision: int = _lib.FJB_FP64, threshold: float = 0.0) -> None:
        """Record the batched build as one CUDA graph under `key`."""
        import torch
        self.build_merged(precision, threshold)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.build_merged(precision, threshold)
        self.graphs[key] = g

    def merged_stats(self) -> dict:
        """The last batched build: device ms of its class launches, the
        class launches and the work units."""
        L = _lib.load()
        ms, nc, nu = C.c_double(), C.c_int64(), C.c_int64()
        rc = L.fjb_batch_stats(self._merged(), C.byref(ms), C.byref(nc), C.byref(nu))
        if rc:
            raise RuntimeError(f"fjb_batch_stats: {L.fjb_batch_last_error(self._batch).decode()}")
        return {"ms": ms.value, "class_launches": nc.value, "units": nu.value}

    def close(self) -> None:
        if self._batch is not None:
            _lib.load().fjb_batch_destroy(self._batch)
            self._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
