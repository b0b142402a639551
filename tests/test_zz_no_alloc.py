"""fjb_fock_build_noalloc: the build for callers that cannot allocate device
memory while their SCF loop runs (a host framework that owns all device
memory through its own pool, or a loop that must not pay for or risk an
allocation between iterations).  Called through the C ABI, twice in a row,
against fjb_fock_build on the same plan and density; the tolerance is the
plain FP64 path's (1e-11 max-abs), the two differing only in the order of
their FP64 atomic additions.  Named to be collected last."""

import ctypes as C

import numpy as np
import pytest

from felizjueves_b200 import _lib, configs
from felizjueves_b200.fock import FockEngine

pytestmark = pytest.mark.gpu


def test_noalloc_build_matches_fock_build_twice(cuda, lib_built):
    import torch
    w = configs.cluster(2, 3)  # s..f shells: every class to (ff|ff)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    J, K, G = eng.build(D)
    torch.cuda.synchronize()
    L = _lib.load()
    st = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for _ in range(2):  # the second call sees the first call's scratch
        J2, K2, G2 = (torch.full_like(J, np.nan) for _ in range(3))
        _lib.check(L.fjb_fock_build_noalloc(eng._h, D.data_ptr(), J2.data_ptr(),
                                            K2.data_ptr(), G2.data_ptr(), st), eng._h)
        torch.cuda.synchronize()
        for a, b in ((J2, J), (K2, K), (G2, G)):
            assert float((a - b).abs().max()) <= 1e-11


def test_noalloc_refuses_sizes_beyond_its_scratch(cuda, lib_built):
    import torch
    w = configs.cluster(20, 3)  # 620 AO > 512
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    out = torch.empty_like(D)
    rc = _lib.load().fjb_fock_build_noalloc(eng._h, D.data_ptr(), out.data_ptr(),
                                            out.data_ptr(), out.data_ptr(), None)
    assert rc == -4
    assert b"exceed its fixed scratch" in _lib.load().fjb_last_error(eng._h)


def test_noalloc_build_matches_oracle(cuda, lib_built, oracle_lib):
    """The no-allocation build held directly to the oracle (3-atom cluster,
    every class to (ff|ff), unscreened), at the plain FP64 bar."""
    import torch
    w = configs.cluster(3, 5)
    eng = FockEngine(w.basis)
    eng.plan(w.D, 0.0, 4)
    D = torch.tensor(w.D, device=cuda)
    J, K, G = (torch.full_like(D, np.nan) for _ in range(3))
    st = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    _lib.check(_lib.load().fjb_fock_build_noalloc(eng._h, D.data_ptr(), J.data_ptr(), K.data_ptr(),
                                                  G.data_ptr(), st), eng._h)
    torch.cuda.synchronize()
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(J.cpu().numpy() - Jo).max() <= 1e-11
    assert np.abs(K.cpu().numpy() - Ko).max() <= 1e-11
    assert np.abs(G.cpu().numpy() - (Jo - 0.5 * Ko)).max() <= 1e-11
