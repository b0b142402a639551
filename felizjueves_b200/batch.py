"""Uneven batched builds: many molecules, one captured launch sequence.

Each molecule keeps its own handle, plan and device buffers (D, J, K, G);
`BatchBuilder.capture` records every molecule's build -- all its class
launches, in FP64 or routed with the learned router -- into ONE CUDA graph,
so a batch is one graph launch with no host work between molecules.  Each
molecule's build events are graph nodes too, so its device time is read back
after every replay (`device_ms`).  The classes of different molecules are
separate launches inside the graph (each kernel is fed one molecule's work
queue); a single persistent kernel over a merged class-sorted queue of all
molecules is not what this does.
"""

from __future__ import annotations

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
