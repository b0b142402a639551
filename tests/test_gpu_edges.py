"""Edge cases of the G build on the GPU: the smallest basis, a closed form, a
density of zeros, a plan with no launches, ragged contraction degrees up to
the staging cap, atoms far apart.  Every result goes through the C ABI and
is held to the oracle (or to an exact value) at the plain FP64 bar: 1e-11
absolute, or 1e-13 of the largest |J|, |K| element where that is above 100
(unnormalised contractions of many primitives give elements of a few
hundred, whose last bits alone are 1e-14)."""

import math

import numpy as np
import pytest

from felizjueves_b200 import _lib
from felizjueves_b200.fock import FockEngine
from felizjueves_b200.shell import Basis, Shell

pytestmark = pytest.mark.gpu

FP64_ABS = 1e-11


def _sym(n, seed):
    A = np.random.default_rng(seed).normal(size=(n, n))
    return (A + A.T) / n


def _vs_oracle(oracle_lib, B, D, tau=0.0):
    eng = FockEngine(B)
    eng.plan(D, tau, 4)
    J, K, G = eng.build_host(D)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(B), D)
    tol = max(FP64_ABS, 1e-13 * max(np.abs(Jo).max(), np.abs(Ko).max()))
    assert np.abs(J - Jo).max() <= tol
    assert np.abs(K - Ko).max() <= tol
    assert np.abs(G - (Jo - 0.5 * Ko)).max() <= tol
    return eng, (J, K, G)


def test_one_s_primitive_closed_form(cuda, lib_built, oracle_lib):
    """One s primitive of exponent a, normalised by its coefficient:
    (ss|ss) = 2 sqrt(a / pi), so J = K = (ss|ss) D and G = (ss|ss) D / 2."""
    from felizjueves_b200.shell import primitive_norm
    a, d = 1.3, 0.7
    B = Basis((Shell(0, (0.2, -0.1, 0.4), [a], [primitive_norm(0, a)]),))
    D = np.array([[d]])
    _, (J, K, G) = _vs_oracle(oracle_lib, B, D)
    v = 2.0 * math.sqrt(a / math.pi)
    assert abs(J[0, 0] - v * d) <= 1e-14 and abs(K[0, 0] - v * d) <= 1e-14
    assert abs(G[0, 0] - 0.5 * v * d) <= 1e-14


def test_ragged_degrees_to_the_staging_cap(cuda, lib_built, oracle_lib):
    """Contraction degrees 1, 2, 5 and 11 on four centres, l = 0..3: pair
    degrees from 1 to 121 (the cap is 128) in one build, unscreened."""
    ex = list(np.geomspace(0.1, 50.0, 11))
    B = Basis((
        Shell(1, (0.0, 0.0, 0.0), ex, list(np.linspace(0.2, 1.0, 11))),
        Shell(0, (1.2, 0.3, -0.4), ex, list(np.linspace(1.0, 0.1, 11))),
        Shell(3, (0.0, 1.5, 0.2), [0.9, 2.5], [0.6, 0.5]),
        Shell(2, (-1.1, 0.2, 0.9), [0.4, 1.1, 3.0, 7.5, 20.0], [0.2, 0.3, 0.4, 0.3, 0.1]),
        Shell(0, (-1.1, 0.2, 0.9), [0.3], [1.0]),
    ))
    _vs_oracle(oracle_lib, B, _sym(B.n_ao, 3))


def test_atoms_far_apart(cuda, lib_built, oracle_lib):
    """Two atoms 150 bohr apart: the cross exchange blocks vanish to
    underflow and the Coulomb coupling is the point-charge tail."""
    sh = []
    for c in ((0.0, 0.0, 0.0), (150.0, 0.0, 0.0)):
        sh += [Shell(0, c, [0.5, 2.0], [0.7, 0.4]), Shell(1, c, [0.8], [1.0]), Shell(2, c, [1.1], [1.0])]
    B = Basis(tuple(sh))
    _vs_oracle(oracle_lib, B, _sym(B.n_ao, 5), tau=1e-12)


@pytest.mark.parametrize("tau", [0.0, 1e-12])
def test_zero_density_gives_exact_zeros(cuda, lib_built, tau):
    import torch
    from felizjueves_b200 import configs
    w = configs.cluster(3, 5)
    D = np.zeros_like(w.D)
    eng = FockEngine(w.basis)
    eng.plan(D, tau, 4)
    Dt = torch.zeros((w.n_ao, w.n_ao), dtype=torch.float64, device=cuda)
    for prec, thr in ((_lib.FJB_FP64, 0.0), (_lib.FJB_ROUTED, 1e-9), (_lib.FJB_FP64_SCATTER, 0.0)):
        J, K, G = eng.build(Dt, precision=prec, threshold=thr)
        torch.cuda.synchronize()
        for X in (J, K, G):
            assert int(torch.count_nonzero(X)) == 0


def test_plan_without_launches(cuda, lib_built):
    """tau above every pair bound: the pre-launch screen drops every batch
    pair, no class kernel runs, and J = K = G = 0 exactly (eager, graph and
    host-buffer builds)."""
    import torch
    from felizjueves_b200 import configs
    w = configs.c0()
    eng = FockEngine(w.basis)
    P = eng.plan(w.D, 1e3, 4)
    assert len(P.launches) == 0
    Dt = torch.tensor(w.D, device=cuda)
    J, K, G = eng.build(Dt)
    torch.cuda.synchronize()
    assert all(int(torch.count_nonzero(X)) == 0 for X in (J, K, G))
    out = [torch.full_like(Dt, 7.0) for _ in range(3)]
    eng.build(Dt, J=out[0], K=out[1], G=out[2], graph=True)
    torch.cuda.synchronize()
    assert all(int(torch.count_nonzero(X)) == 0 for X in out)
    Jh, Kh, Gh = eng.build_host(w.D)
    assert not Jh.any() and not Kh.any() and not Gh.any()


def test_spherical_build_matches_oracle(cuda, lib_built, oracle_lib):
    """A spherical density through SphericalFock: J, K, G in real solid
    harmonics against T^T (oracle's Cartesian J, K) T."""
    import torch
    from felizjueves_b200 import configs
    from felizjueves_b200.spherical import SphericalFock, transform
    w = configs.cluster(3, 5)
    T = transform(w.basis)
    ns = T.shape[1]
    Ds = _sym(ns, 9)
    sf = SphericalFock(w.basis)
    sf.plan(Ds, 0.0, 4)
    J, K, G = (M.cpu().numpy() for M in sf.build(torch.tensor(Ds, device=cuda)))
    Dc = T @ Ds @ T.T
    Dc = 0.5 * (Dc + Dc.T)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), Dc)
    assert np.abs(J - T.T @ Jo @ T).max() <= FP64_ABS
    assert np.abs(K - T.T @ Ko @ T).max() <= FP64_ABS
    assert np.abs(G - T.T @ (Jo - 0.5 * Ko) @ T).max() <= FP64_ABS
