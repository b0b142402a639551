"""The tabulated Rys rule (felizjueves_b200/csrc/rys_rule.h, rys_table.cpp),
the quadrature a device Rys VRR reads, evaluated on the host by
tests/rys_harness.cpp: the Boys moments sum_n w_n x_n^m = F_m(T) for
m <= 2n - 1 to 1e-14 relative (n = 1..7, T from 0 to 1e5, across the
table's switch at T = 128), the reference's own fp64 rule (rys/roots.py,
n <= 5) to 1e-13, and the oracle's rule to 1e-12."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import golden

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = tmp_path_factory.mktemp("rys") / "rys_harness"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "felizjueves_b200", "csrc"),
                    os.path.join(REPO, "tests", "rys_harness.cpp"),
                    os.path.join(REPO, "felizjueves_b200", "csrc", "rys_table.cpp"), "-o", str(exe)], check=True)

    def rule(pairs):
        lines = "".join(f"{int(n)} {float(T)!r}\n" for n, T in pairs)
        out = subprocess.run([str(exe)], input=lines, capture_output=True, text=True, check=True).stdout
        res = []
        for line in out.strip().split("\n"):
            v = [float(s) for s in line.split()[1:]]
            res.append((np.array(v[0::2]), np.array(v[1::2])))
        return res
    return rule


TS = [0.0, 1e-10, 1e-3, *np.linspace(0.01, 140.0, 211), 127.999, 128.0, 128.001, 200.0, 1e3, 1e5]


def test_moments(harness, oracle_lib):
    from oracle import oracle
    pairs = [(n, T) for n in range(1, 8) for T in TS]
    for (n, T), (x, w) in zip(pairs, harness(pairs)):
        assert len(x) == n and np.all(np.diff(x) > 0) and np.all(w > 0)
        for m in range(2 * n):
            F = oracle.boys(m, T)
            assert abs(float((w * x ** m).sum()) - F) <= 1e-14 * F, (n, T, m)


def test_matches_reference_and_oracle(harness):
    from oracle import rys
    z = golden("rys_roots.npz")
    pairs = [(n, T) for n in range(1, 6) for T in z["T"]]
    for (n, T), (x, w) in zip(pairs, harness(pairs)):
        k = list(z["T"]).index(T)
        xr, wr = z["x"][n - 1, k, :n], z["w"][n - 1, k, :n]
        assert np.abs(x - xr).max() <= 1e-13 * np.abs(xr).max()
        assert np.abs(w - wr).max() <= 1e-13 * np.abs(wr).max()
    pairs = [(7, T) for T in TS]
    for (n, T), (x, w) in zip(pairs, harness(pairs)):
        xo, wo = rys.roots_weights(n, T)
        assert np.abs(x - xo).max() <= 1e-12 * np.abs(xo).max()
        assert np.abs(w - wo).max() <= 1e-12 * np.abs(wo).max()


def test_rys_boundary_with_hgp_hrr_matches_oracle(oracle_lib, tmp_path):
    """The Rys boundary (csrc/rys_vrr.h) fed to the HGP class's own HRR
    tables gives the oracle's ERI blocks (26 canonical quartets of a cluster
    with shells to l = 3, (ff|ff) among them): 1e-11 of the block's largest
    element (the HRR's |AB|^k cancellation leaves ~1e-12)."""
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    from felizjueves_b200 import configs
    from oracle import oracle
    exe = tmp_path / "rys_q"
    c = os.path.join(REPO, "felizjueves_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", c, "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "rys_quartet_harness.cpp"), os.path.join(c, "rys_table.cpp"),
                    os.path.join(c, "hgp_tables.cpp"), "-o", str(exe)], check=True)
    B = configs.cluster(3, 5).basis
    ob = oracle.OracleBasis.of(B)
    sh = B.shells

    def canon(q):
        a, b, cc, d = q
        if sh[a].l > sh[b].l:
            a, b = b, a
        if sh[cc].l > sh[d].l:
            cc, d = d, cc
        if (sh[a].l, sh[b].l) > (sh[cc].l, sh[d].l):
            a, b, cc, d = cc, d, a, b
        return [a, b, cc, d]

    rng = np.random.default_rng(1)
    qs = [canon([int(v) for v in rng.integers(0, len(sh), 4)]) for _ in range(25)]
    fs = [i for i, s in enumerate(sh) if s.l == 3][:2]
    qs.append([fs[0], fs[1], fs[0], fs[1]])
    for q in qs:
        inp = "".join(f"{sh[i].l} {float(sh[i].centre[0])!r} {float(sh[i].centre[1])!r} "
                      f"{float(sh[i].centre[2])!r} {sh[i].n_prim} "
                      + " ".join(repr(float(x)) for x in sh[i].exponents) + " "
                      + " ".join(repr(float(x)) for x in sh[i].coefficients) + "\n" for i in q)
        out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True)
        r = np.array([float(v) for v in out.stdout.split()])
        m = oracle.eri_block(ob, *q)
        assert np.abs(r - m).max() <= 1e-11 * np.abs(m).max(), q
