"""GPU parity: the sm_100a kernels through the C ABI against the oracle, the
reference's recorded outputs and the libcint fixtures.

Tolerances (stated, not tuned):
  Boys           1e-13 relative to the reference's quadrature
                 (test/test_eval_boys_device.py:16-18 BOYS_REL)
  ERI blocks     1e-12 of the block's absolute-value twin `scale`
                 (eri/eri.py:133, the reference's per-ERI bar)
  J, K, G FP64   1e-11 max-abs against the oracle (the plain FP64 bar)
  libcint        1e-12 of max |vj|, max |vk|
  screen mask    bit-exact
"""

import ctypes as C

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine
from felizjueves_b200.shell import Basis, Shell

pytestmark = pytest.mark.gpu

FP64_ABS = 1e-11


def _basis_from_npz(g):
    shells = []
    for s in range(len(g["l"])):
        p0, n = int(g["prim0"][s]), int(g["nprim"][s])
        shells.append(Shell(int(g["l"][s]), tuple(g["centre"][s]), g["exps"][p0:p0 + n],
                            g["coefs"][p0:p0 + n]))
    return Basis(tuple(shells))


def test_boys_device_matches_reference(cuda, lib_built):
    import torch
    from felizjueves_b200 import _lib
    z = golden("boys_ref.npz")
    T = torch.tensor(z["T"], dtype=torch.float64, device=cuda)
    M = 18
    F = torch.zeros(len(z["T"]) * (M + 1), dtype=torch.float64, device=cuda)
    _lib.check(_lib.load().fjb_boys(M, T.data_ptr(), len(z["T"]), F.data_ptr()))
    got = F.cpu().numpy().reshape(-1, M + 1).T
    ref = z["F"][: M + 1]
    rel = np.abs(got - ref) / np.abs(ref)
    assert rel.max() < 1e-13, rel.max()


@pytest.mark.parametrize("wname", ["c0", "c1"])
def test_eri_tap_matches_reference(cuda, lib_built, wname):
    """The HGP tap against the reference's MMD eri_block.  The two
    recurrences cancel differently, so an element is held to 1e-12 of its
    own `scale` or, for elements that vanish against their block (a far
    pair's HRR multiplies by |AB|^l: the (sp|sf) quartet (200,68|168,463)
    of the 64-atom cluster, with |(ab|cd)| ~ 1e-24, misses 1e-11 of its
    block's scale by 0.2%), to 1e-10 of the block's largest `scale` -- both
    far below anything a J/K/G element can see."""
    w = getattr(configs, wname)()
    z = golden(f"eri_{wname}.npz")
    eng = FockEngine(w.basis)
    blocks = eng.eri_blocks(z["quartets"])
    worst = 0.0
    for i, q in enumerate(z["quartets"]):
        lo, hi = z["offsets"][i], z["offsets"][i + 1]
        sc = z["scale"][lo:hi]
        err = np.abs(blocks[i].ravel() - z["values"][lo:hi])
        tol = np.maximum(1e-12 * sc, 1e-10 * sc.max())
        worst = max(worst, float((err / np.maximum(tol, 1e-300)).max()))
        assert np.all(err <= tol), (tuple(q), err.max(), sc.max())
    print(f"worst err/tol = {worst:.3f}")


def _gpu_jkg(basis, D, tau, n=4):
    eng = FockEngine(basis)
    eng.plan(D, tau, n)
    return eng, eng.build_host(D)


def test_c0_fp64_matches_oracle_unscreened(cuda, lib_built, oracle_lib):
    w = configs.c0()
    _, (J, K, G) = _gpu_jkg(w.basis, w.D, 0.0)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(J - Jo).max() <= FP64_ABS
    assert np.abs(K - Ko).max() <= FP64_ABS
    assert np.abs(G - (Jo - 0.5 * Ko)).max() <= FP64_ABS


def test_c0_screened_build_close_to_oracle(cuda, lib_built, oracle_lib):
    """At tau = 1e-12 every skipped term is < tau by the proved bounds; the
    whole-matrix effect stays orders below the 1e-8 mixed-precision budget."""
    w = configs.c0()
    _, (J, K, G) = _gpu_jkg(w.basis, w.D, w.tau, w.n_mag)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(G - (Jo - 0.5 * Ko)).max() <= 1e-9


def test_c0_matches_reference_host_path(cuda, lib_built):
    """The 6-atom workload against the reference's own host path run on it
    at its tau, 1e-12 (coulomb_matrix + exchange_matrix, the J and K the
    reference computes in 1,900 s and 2,851 s on one core;
    tests/golden/make_golden.py part_cpu_c0).  The two screens differ (the
    reference's sorted J break and K continue against the six-block screen),
    each dropping only terms below tau by its bounds: held to 1e-9."""
    w = configs.c0()
    z = golden("cpu_c0.npz")
    _, (J, K, G) = _gpu_jkg(w.basis, w.D, w.tau, w.n_mag)
    assert np.abs(J - z["J"]).max() <= 1e-9
    assert np.abs(K - z["K"]).max() <= 1e-9
    assert np.abs(G - z["G"]).max() <= 1e-9


def test_c0_screen_mask_bit_exact(cuda, lib_built):
    w = configs.c0()
    z = golden("screen_c0.npz")
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    m = eng.screen_mask(w.D)
    assert len(m) == len(z["rows"])
    assert np.array_equal(m, z["rows"][:, 3].astype(np.uint8))


def test_c1_screen_mask_bit_exact_on_sample(cuda, lib_built):
    """The 64-atom cluster's six-block mask (1.34e9 launched quartets) on the
    reference's walk_f prediction for 16,800 sampled launched quartets: per
    (class, K_AB, K_CD) key the 12 of 400 draws whose bound lies nearest tau
    and 8 at random (tests/golden/make_golden.py part_screen_c1)."""
    w = configs.c1()
    z = golden("screen_c1_sample.npz")
    eng = FockEngine(w.basis)
    P = eng.plan(w.D, w.tau, w.n_mag)
    assert P.quartets_launched == int(z["n_launched"])
    qbase, q = [], 0
    for L in P.launches:
        nb, nk = len(P.batches[L.bra].pairs), len(P.batches[L.ket].pairs)
        qbase.append(q)
        q += nb * (nb + 1) // 2 if L.bra == L.ket else nb * nk
    rows = z["rows"].astype(np.int64)
    li, ib, ik = rows[:, 0], rows[:, 1], rows[:, 2]
    n_ket = np.asarray([len(P.batches[P.launches[i].ket].pairs) for i in li], np.int64)
    diag = np.asarray([P.launches[i].bra == P.launches[i].ket for i in li])
    row = np.where(diag, ib * n_ket - ib * (ib - 1) // 2 - ib, ib * n_ket)
    at = np.asarray(qbase, np.int64)[li] + row + ik
    m = eng.screen_mask(w.D, at=at)
    assert np.array_equal(m, rows[:, 3].astype(np.uint8)), int((m != rows[:, 3]).sum())


LIBCINT = ["h2_sto3g", "h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "h10_chain_ccpvdz", "co_ccpvtz"]


@pytest.mark.parametrize("name", LIBCINT)
def test_jk_matches_libcint(cuda, lib_built, name):
    g = golden(f"libcint_{name}.npz")
    B = _basis_from_npz(g)
    _, (J, K, G) = _gpu_jkg(B, g["D"], 0.0)
    assert np.abs(J - g["vj"]).max() <= 1e-12 * np.abs(g["vj"]).max()
    assert np.abs(K - g["vk"]).max() <= 1e-12 * np.abs(g["vk"]).max()
    assert np.abs(G - (g["vj"] - 0.5 * g["vk"])).max() <= 1e-12 * np.abs(g["vj"]).max()


def test_exchange_matrix_matches_libcint(cuda, lib_built):
    """The reference-shaped K driver (eri/k_exchange/k.py:482) on libcint."""
    from felizjueves_b200.fock import exchange_matrix
    g = golden("libcint_co_ccpvtz.npz")
    K = exchange_matrix(_basis_from_npz(g), g["D"])
    assert np.abs(K - g["vk"]).max() <= 1e-12 * np.abs(g["vk"]).max()


@pytest.mark.parametrize("name,atoms,wfn", [("c0_1at", 1, "c0"), ("c0_2at", 2, "c0"),
                                            ("c1_1at", 1, "c1")])
def test_jk_matches_reference_host_path(cuda, lib_built, name, atoms, wfn):
    w = configs.sub_workload(getattr(configs, wfn)(), atoms)
    g = golden(f"jk_{name}.npz")
    _, (J, K, G) = _gpu_jkg(w.basis, w.D, 0.0)
    assert np.abs(J - g["J"]).max() <= FP64_ABS
    assert np.abs(K - g["K"]).max() <= FP64_ABS


@pytest.mark.parametrize("atoms,seed", [(3, 5), (4, 5)])
def test_cluster_fp64_matches_oracle(cuda, lib_built, oracle_lib, atoms, seed):
    """Every class to (ff|ff) at once, unscreened."""
    w = configs.cluster(atoms, seed)
    _, (J, K, G) = _gpu_jkg(w.basis, w.D, 0.0)
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(J - Jo).max() <= FP64_ABS
    assert np.abs(K - Ko).max() <= FP64_ABS
    assert np.abs(G - (Jo - 0.5 * Ko)).max() <= FP64_ABS


@pytest.mark.parametrize("atoms,seed", [(3, 5), (4, 7)])
def test_routed_build_within_budget(cuda, lib_built, oracle_lib, atoms, seed):
    """The routed build (FP32 recurrences for quartets under the 1e-9
    Schwarz x |D| bound) stays within the metric's budget max|dG| <= 1e-8
    against the FP64 build and against the oracle; the error is reported."""
    import torch
    from felizjueves_b200 import _lib
    w = configs.cluster(atoms, seed)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    G64 = eng.build(D)[2].clone()
    G32 = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-9)[2].clone()
    torch.cuda.synchronize()
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    d64 = float((G32 - G64).abs().max())
    dor = float(np.abs(G32.cpu().numpy() - (Jo - 0.5 * Ko)).max())
    print(f"routed: max|dG| vs FP64 {d64:.3e}, vs oracle {dor:.3e}")
    assert d64 <= 1e-8 and dor <= 1e-8


def test_all_fp32_build_at_fp32_accuracy(cuda, lib_built):
    """With a routing threshold above every bound, every unit of every class
    runs an FP32 kernel (the register bodies and, for the classes without
    one, the interpreter in FP32): G then agrees with the FP64 build to FP32
    accuracy, relative to G's size."""
    import torch
    from felizjueves_b200 import _lib, router
    w = configs.cluster(3, 5)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    G64 = eng.build(D)[2].clone()
    G32 = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e30)[2].clone()
    torch.cuda.synchronize()
    n32, n64 = router.route_stats(eng)
    rel = float((G32 - G64).abs().max() / G64.abs().max())
    print(f"all-FP32 build: {n32} FP32 units, {n64} FP64; max|dG|/max|G| {rel:.2e}")
    assert n64 == 0 and n32 > 0
    assert rel <= 1e-5


def test_graph_build_replays_the_build(cuda, lib_built):
    """The captured build equals the direct one, and replaying it after D is
    updated in place gives the new density's result (the SCF-loop use)."""
    import torch
    from felizjueves_b200 import _lib
    w = configs.cluster(2, 3)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    D2 = torch.tensor(configs.perturbed_density(w.D, 3), device=cuda)
    for prec in (_lib.FJB_FP64, _lib.FJB_ROUTED):
        ref1 = [t.clone() for t in eng.build(D, precision=prec)]
        ref2 = [t.clone() for t in eng.build(D2, precision=prec)]
        Dw = D.clone()
        out = [torch.empty_like(D) for _ in range(3)]
        eng.build(Dw, J=out[0], K=out[1], G=out[2], precision=prec, graph=True)
        torch.cuda.synchronize()
        for a, b in zip(out, ref1):
            assert float((a - b).abs().max()) <= 1e-11
        Dw.copy_(D2)
        eng.build(Dw, J=out[0], K=out[1], G=out[2], precision=prec, graph=True)
        torch.cuda.synchronize()
        for a, b in zip(out, ref2):
            assert float((a - b).abs().max()) <= 1e-11
        # the build and class timings read after a replay are that replay's
        ms, n_launches = eng.last_build_stats()
        assert ms > 0.0 and n_launches > 0
        assert all(r["ms"] >= 0.0 for r in eng.class_stats())


def test_device_build_matches_host_build(cuda, lib_built):
    import torch
    w = configs.c0()
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    Jh, Kh, Gh = eng.build_host(w.D)
    D = torch.tensor(w.D, device=cuda)
    J, K, G = eng.build(D)
    torch.cuda.synchronize()
    for a, b in ((J, Jh), (K, Kh), (G, Gh)):
        assert np.abs(a.cpu().numpy() - b).max() <= 1e-12


@pytest.mark.slow
def test_c1_full_size_properties(cuda, lib_built):
    """At full size the oracle cannot run; size-independent properties hold:
    exact symmetry of J, K, G; repeatability; linearity in D within the
    screen's bound."""
    import torch
    w = configs.c1()
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    J, K, G = eng.build(D)
    J2, K2, G2 = eng.build(D)
    torch.cuda.synchronize()
    for M in (J, K, G):
        assert torch.equal(M, M.T)
    s = float(G.abs().max())
    assert float((G - G2).abs().max()) <= 1e-13 * s
    D2 = torch.tensor(configs.perturbed_density(w.D, 0), device=cuda) - D
    Ga = eng.build(D + D2)[2]
    Gb = eng.build(D2)[2]
    torch.cuda.synchronize()
    assert float((Ga - G - Gb).abs().max()) <= 1e-8


def test_refuses_asymmetric_density(cuda, lib_built):
    w = configs.c0()
    eng = FockEngine(w.basis)
    D = w.D.copy()
    D[2, 5] *= 1 + 1e-15
    with pytest.raises(ValueError, match="not symmetric"):
        eng.plan(D, w.tau, 4)


@pytest.mark.parametrize("name", ["h2_sto3g", "h2o_sto3g", "h2o_631g"])
def test_schwarz_diagonal_matches_libcint(cuda, lib_built, name):
    """(mn|mn) of every AO pair (eri/schwarz.py:86-102) against libcint's
    int2e diagonal the reference tracks; Q = sqrt(max(., 0))."""
    from felizjueves_b200.fock import diagonal_matrix, schwarz_matrix
    g = golden(f"libcint_{name}_schwarz.npz")
    B = _basis_from_npz(g)
    M = diagonal_matrix(B)
    ref = g["int2e_diag"]
    assert np.abs(M - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.array_equal(M, M.T)
    Q = schwarz_matrix(B)
    assert np.allclose(Q, np.sqrt(np.maximum(ref, 0.0)), rtol=1e-11, atol=1e-14)


@pytest.mark.parametrize("wname,tau", [("c0", 0.0), ("cluster3", 0.0), ("c0", 1e-12)])
def test_atomics_free_build_reproducible(cuda, lib_built, oracle_lib, wname, tau):
    """FJB_FP64_SCATTER (the reference's scatter lever: slots, then an ordered
    per-element sum) gives the same J, K, G as the atomic build to rounding,
    the oracle's within 1e-11 when unscreened, and the same bits on every
    build (the property atomics do not have)."""
    import torch
    from felizjueves_b200 import _lib
    w = configs.by_name(wname)
    eng = FockEngine(w.basis)
    eng.plan(w.D, tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    ref = [t.clone() for t in eng.build(D)]
    runs = [[t.clone() for t in eng.build(D, precision=_lib.FJB_FP64_SCATTER)] for _ in range(3)]
    torch.cuda.synchronize()
    for r in runs[1:]:
        for a, b in zip(r, runs[0]):
            assert torch.equal(a, b)  # bit-identical
    for a, b in zip(runs[0], ref):
        assert float((a - b).abs().max()) <= 1e-12
    if tau == 0.0:
        Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
        J, K, G = (t.cpu().numpy() for t in runs[0])
        assert np.abs(J - Jo).max() <= FP64_ABS
        assert np.abs(K - Ko).max() <= FP64_ABS
    # graph replay of the same mode
    out = [torch.empty_like(D) for _ in range(3)]
    eng.build(D, J=out[0], K=out[1], G=out[2], precision=_lib.FJB_FP64_SCATTER, graph=True)
    torch.cuda.synchronize()
    for a, b in zip(out, runs[0]):
        assert torch.equal(a, b)


def test_fp32_tap_is_the_routed_arithmetic(cuda, lib_built):
    """fjb_eri_blocks_fp32 (the FP32 recurrences a routed quartet runs)
    agrees with the FP64 tap to FP32 accuracy measured on the whole sample,
    while single quartets can lose digits to cancellation (the HRR's |AB|^k
    factors): the spread is reported."""
    w = configs.c0()
    z = golden("eri_c0.npz")
    eng = FockEngine(w.basis)
    b64 = eng.eri_blocks(z["quartets"])
    b32 = eng.eri_blocks(z["quartets"], fp32=True)
    err = np.array([np.abs(x - y).max() for x, y in zip(b32, b64)])
    mag = np.array([np.abs(y).max() for y in b64])
    big = max(mag)
    rel = err[mag > 0] / mag[mag > 0]
    print(f"FP32 tap: max|d|/max|ERI| {err.max() / big:.2e}; per-quartet relative error "
          f"median {np.median(rel):.1e}, 99th percentile {np.percentile(rel, 99):.1e}")
    assert np.all(np.isfinite(err))
    assert err.max() <= 1e-5 * big
