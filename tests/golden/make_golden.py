"""Generate the golden fixtures under tests/golden/ from the reference.

This script is test infrastructure. It imports the reference's own Python
(`src/felizjueves`, pure Python + numpy) from a reference checkout and
records its outputs on this repository's seeded workloads, plus the
libcint/PySCF fixtures the reference tracks (`test/oracle/fixtures/*.json`).
Nothing at test time reads the reference: the tests read only the .npz/.json
files this script writes.

    python tests/golden/make_golden.py --ref /path/to/reference [parts...]

parts: libcint eri_libcint numeric_j numeric_metric boys eri eri_c1_sample plan_c0 plan_c1 jk_small cpu_c0 screen_c0 screen_c1 cost jplan_c0 jplan_c1 scatter_c0 scatter_c1 onee
scf bse harmonics grad rys hjk_c0 boys_zero (default: all
but plan_c1, jk_small, eri_c1_sample and jplan_c1, which take minutes).
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import sys
import time
from functools import partial

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

REF = os.environ.get("FJB_REF")  # set in main; inherited by spawned workers
if REF:
    sys.path.insert(0, os.path.join(REF, "src"))


def _ref_imports():
    p = os.path.join(os.environ["FJB_REF"], "src")
    if p not in sys.path:
        sys.path.insert(0, p)


def ref_basis(basis):
    from felizjueves.ao.shell import Basis, Shell
    return Basis(tuple(Shell(s.l, s.centre, s.exponents, s.coefficients)
                       for s in basis.shells))


def flat_shells(shells_l, centres, exps, coefs):
    n = len(shells_l)
    p0, npr, ex, co = [], [], [], []
    for e, c in zip(exps, coefs):
        p0.append(len(ex))
        npr.append(len(e))
        ex.extend(e)
        co.extend(c)
    return dict(l=np.asarray(shells_l, np.int32),
                centre=np.asarray(centres, np.float64).reshape(n, 3),
                prim0=np.asarray(p0, np.int32), nprim=np.asarray(npr, np.int32),
                exps=np.asarray(ex, np.float64),
                coefs=np.asarray(co, np.float64))


# --- libcint fixtures ---------------------------------------------------------

LIBCINT = ["h2_sto3g", "h2o_sto3g", "h2o_631g", "h2o_ccpvdz", "h10_chain_ccpvdz",
           "co_ccpvtz"]


def part_libcint():
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for name in LIBCINT:
        dj = json.load(open(os.path.join(fx, name + "_j.json")))
        dk = json.load(open(os.path.join(fx, name + "_k.json")))
        assert dj["provenance"]["cart"] is True
        conv = dj["converted"]["shells"]
        assert conv == dk["converted"]["shells"]
        n = dj["nao"]
        D = np.asarray(dj["arrays"]["density"]["values"]).reshape(n, n)
        Dk = np.asarray(dk["arrays"]["density"]["values"]).reshape(n, n)
        assert np.array_equal(D, Dk)
        vj = np.asarray(dj["arrays"]["vj"]["values"]).reshape(n, n)
        vk = np.asarray(dk["arrays"]["vk"]["values"]).reshape(n, n)
        sh = flat_shells([s["l"] for s in conv], [s["centre"] for s in conv],
                         [s["exponents"] for s in conv],
                         [s["coefficients"] for s in conv])
        np.savez_compressed(os.path.join(HERE, f"libcint_{name}.npz"),
                            D=D, vj=vj, vk=vk, **sh,
                            source=np.asarray(f"test/oracle/fixtures/{name}_j.json "
                                              f"+ _k.json (PySCF "
                                              f"{dj['provenance']['pyscf']}, libcint "
                                              f"{dj['provenance']['libcint']})"))
        print("libcint", name, n)
    for name in ("h2_sto3g", "h2o_sto3g", "h2o_631g"):
        ds = json.load(open(os.path.join(fx, name + "_schwarz.json")))
        assert ds["provenance"]["cart"] is True
        conv = ds["converted"]["shells"]
        n = ds["nao"]
        diag = np.asarray(ds["arrays"]["int2e_diag"]["values"]).reshape(n, n)
        sh = flat_shells([s["l"] for s in conv], [s["centre"] for s in conv],
                         [s["exponents"] for s in conv],
                         [s["coefficients"] for s in conv])
        np.savez_compressed(os.path.join(HERE, f"libcint_{name}_schwarz.npz"),
                            int2e_diag=diag, **sh,
                            source=np.asarray(f"test/oracle/fixtures/{name}_schwarz.json"))
        print("libcint schwarz", name, n)


ERI_LIBCINT = ["h2o_631g_eri", "hf_ccpvtz_eri", "hf_ccpvtz_eri_l9", "hf_ccpvtz_eri_l10",
               "hf_ccpvtz_eri_l11", "hf_ccpvtz_eri_l12"]


def part_eri_libcint():
    """libcint's Cartesian (ij|kl) blocks the reference tracks
    (`int2e:i,j,k,l` arrays, one shell quartet per class: every class to
    (ff|ff) over the hf_ccpvtz files), with the converted shells they
    index."""
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for name in ERI_LIBCINT:
        d = json.load(open(os.path.join(fx, name + ".json")))
        assert d["provenance"]["cart"] is True
        conv = d["converted"]["shells"]
        qs, vals, offs = [], [], [0]
        for key, arr in d["arrays"].items():
            if not key.startswith("int2e:"):
                continue
            q = tuple(int(x) for x in key[len("int2e:"):].split(","))
            v = np.asarray(arr["values"], np.float64)
            assert tuple(arr["shape"]) == tuple((conv[s]["l"] + 1) * (conv[s]["l"] + 2) // 2
                                                for s in q)
            qs.append(q)
            vals.append(v)
            offs.append(offs[-1] + len(v))
        sh = flat_shells([s["l"] for s in conv], [s["centre"] for s in conv],
                         [s["exponents"] for s in conv], [s["coefficients"] for s in conv])
        np.savez_compressed(os.path.join(HERE, f"libcint_{name}.npz"),
                            quartets=np.asarray(qs, np.int32), values=np.concatenate(vals),
                            offsets=np.asarray(offs, np.int64), **sh,
                            source=np.asarray(f"test/oracle/fixtures/{name}.json (PySCF "
                                              f"{d['provenance']['pyscf']}, libcint "
                                              f"{d['provenance']['libcint']})"))
        print("libcint eri", name, len(qs), "blocks")


# --- one-electron matrices: libcint int1e_* and the reference's own S, T, V ---

ONEE = ["h2_sto3g_j", "h2o_sto3g_j", "h2o_631g_j", "h2o_ccpvdz_j", "h10_chain_ccpvdz_j",
        "hf_ccpvtz", "prim_spd_f", "prim_spdf"]


def _fixture_arrays(d, n, *keys):
    return [np.asarray(d["arrays"][k]["values"]).reshape(n, n) for k in keys]


def part_onee():
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    todo = [(name, [name]) for name in ONEE] + [("co_ccpvtz", ["co_ccpvtz_j_st", "co_ccpvtz_j_vh"])]
    for name, files in todo:
        ds = [json.load(open(os.path.join(fx, f + ".json"))) for f in files]
        for d in ds:
            assert d["provenance"]["cart"] is True and d["provenance"]["mol"]["unit"] == "Bohr"
        conv = ds[0]["converted"]["shells"]
        n = ds[0]["nao"]
        arr = {}
        for d in ds:
            arr.update({k: v for k, v in d["arrays"].items()})
        dd = {"arrays": arr}
        S, T, V, H = _fixture_arrays(dd, n, "int1e_ovlp", "int1e_kin", "int1e_nuc", "hcore")
        atoms = ds[0]["atoms"]
        sh = flat_shells([s["l"] for s in conv], [s["centre"] for s in conv],
                         [s["exponents"] for s in conv],
                         [s["coefficients"] for s in conv])
        np.savez_compressed(os.path.join(HERE, f"onee_{name}.npz"), S=S, T=T, V=V, H=H,
                            charges=np.asarray([a["charge"] for a in atoms], np.float64),
                            coords=np.asarray([a["coord"] for a in atoms], np.float64), **sh,
                            source=np.asarray(" + ".join(f"test/oracle/fixtures/{f}.json" for f in files)
                                              + f" (PySCF {ds[0]['provenance']['pyscf']}, libcint "
                                              f"{ds[0]['provenance']['libcint']})"))
        print("onee", name, n)
    # the reference's own S, T, V on the 3-atom seeded cluster (l to 3),
    # nuclei of charges 3, 1, 2 on its atoms
    from felizjueves.one_electron.kinetic import kinetic_matrix
    from felizjueves.one_electron.overlap import overlap_matrix
    from felizjueves.one_electron.potential import potential_matrix
    from felizjueves.reference.pq import one_centre
    from felizjueves_b200 import configs
    w = configs.cluster(3, 5)
    B = ref_basis(w.basis)
    centres = []
    for sh_ in w.basis.shells:
        if sh_.centre not in centres:
            centres.append(sh_.centre)
    nuclei = [(float(z), c) for z, c in zip((3, 1, 2), centres)]
    S = np.asarray(overlap_matrix(B))
    T = np.asarray(kinetic_matrix(B))
    V = np.asarray(potential_matrix(B, nuclei, one_centre=one_centre))
    np.savez_compressed(os.path.join(HERE, "onee_ref_cluster3.npz"), S=S, T=T, V=V,
                        charges=np.asarray([z for z, _ in nuclei]),
                        coords=np.asarray([c for _, c in nuclei]),
                        source=np.asarray("reference one_electron overlap_matrix, kinetic_matrix, "
                                          "potential_matrix (one_centre from reference/pq.py) on "
                                          "configs.cluster(3, 5)"))
    print("onee reference cluster3", w.basis.n_ao)


# --- converged closed-shell SCF: PySCF's RHF density and orbital energies ----

SCF = ["h2o_sto3g_grad", "h2o_631g_grad", "h2o_ccpvdz_grad", "nh2f_631g_grad"]


def part_scf():
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for name in SCF:
        d = json.load(open(os.path.join(fx, name + ".json")))
        assert d["provenance"]["cart"] is True and d["provenance"]["mol"]["unit"] == "Bohr"
        assert d["provenance"]["mol"]["charge"] == 0 and d["provenance"]["mol"]["spin"] == 0
        conv = d["converted"]["shells"]
        n = d["nao"]
        sh = flat_shells([s["l"] for s in conv], [s["centre"] for s in conv],
                         [s["exponents"] for s in conv],
                         [s["coefficients"] for s in conv])
        atoms = d["atoms"]
        np.savez_compressed(os.path.join(HERE, f"scf_{name.replace('_grad', '')}.npz"),
                            D=np.asarray(d["arrays"]["density"]["values"]).reshape(n, n),
                            mo_energy=np.asarray(d["arrays"]["mo_energy"]["values"]),
                            mo_occ=np.asarray(d["arrays"]["mo_occ"]["values"]),
                            charges=np.asarray([a["charge"] for a in atoms], np.float64),
                            coords=np.asarray([a["coord"] for a in atoms], np.float64), **sh,
                            source=np.asarray(f"test/oracle/fixtures/{name}.json ({d['density_recipe']}; "
                                              f"PySCF {d['provenance']['pyscf']}, libcint "
                                              f"{d['provenance']['libcint']})"))
        print("scf", name, n)


# --- nuclear-gradient J/K terms: libcint int2e_ip1 contracted by PySCF --------

def part_grad():
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for name in SCF:
        d = json.load(open(os.path.join(fx, name + ".json")))
        n = d["nao"]
        arr = d["arrays"]
        g = {k.replace(":", "_"): np.asarray(arr[k]["values"]).reshape(arr[k]["shape"])
             for k in ("vj1", "vk1", "grad:j", "grad:k", "density", "dme", "int1e_ipovlp", "int1e_ipkin",
                       "int1e_ipnuc", "int1e_iprinv", "grad:h", "grad:s", "grad:nuc", "grad:total")}
        ao_atom = [int(lbl.split()[0]) for lbl in d["ao_labels"]]
        np.savez_compressed(os.path.join(HERE, f"grad_{name.replace('_grad', '')}.npz"), **g,
                            ao_atom=np.asarray(ao_atom, np.int32),
                            source=np.asarray(f"test/oracle/fixtures/{name}.json vj1, vk1 (PySCF "
                                              f"grad.rhf.get_jk over int2e_ip1), int1e_ip*, the RHF "
                                              f"gradient's terms, density, dme; PySCF "
                                              f"{d['provenance']['pyscf']}, libcint "
                                              f"{d['provenance']['libcint']}"))
        assert g["vj1"].shape == (3, n, n)
        print("grad", name, n)


# --- the Rys rule: the reference's fp64 nodes and weights ---------------------

def part_rys():
    """rys/roots.py roots_weights(n, T), n = 1..5, on a T grid across its
    switch (T = 80) and out to 1e4."""
    from felizjueves.rys.roots import roots_weights
    Ts = np.concatenate([[0.0, 1e-12, 1e-6], np.geomspace(1e-3, 1e4, 57), [79.9, 80.0, 80.1]])
    x = np.zeros((5, len(Ts), 5))
    w = np.zeros((5, len(Ts), 5))
    for n in range(1, 6):
        for k, T in enumerate(Ts):
            xs, ws = roots_weights(n, float(T))
            x[n - 1, k, :n] = xs
            w[n - 1, k, :n] = ws
    np.savez_compressed(os.path.join(HERE, "rys_roots.npz"), T=Ts, x=x, w=w,
                        source=np.asarray("reference rys/roots.py roots_weights(n, T), n = 1..5"))
    print("rys", len(Ts))


# --- real solid harmonics over Cartesians: the reference's convention ---------

def part_harmonics():
    """The reference's aux_harmonics(l), l = 0..6 (eri/density_fit/
    kernel_eri3.py: columns m = -l..l over cartesians(l))."""
    from felizjueves.eri.density_fit.kernel_eri3 import aux_harmonics
    out = {f"l{l}": np.asarray(aux_harmonics(l)) for l in range(7)}
    np.savez_compressed(os.path.join(HERE, "harmonics.npz"), **out,
                        source=np.asarray("reference eri/density_fit/kernel_eri3.py aux_harmonics(l), "
                                          "l = 0..6, rows m = -l..l"))
    print("harmonics", len(out))


# --- Basis Set Exchange documents: the elements the fixtures use -------------

BSE_SETS = ["sto-3g.json", "6-31g.json", "cc-pVDZ.json", "cc-pVTZ.json"]
BSE_ELEMENTS = ["1", "6", "7", "8", "9"]
BSE_CASES = [("h2_sto3g_j", "sto-3g.json", False), ("h2o_631g_j", "6-31g.json", False),
             ("h2o_ccpvdz_j", "cc-pVDZ.json", True), ("h2o_ccpvdz_j", "cc-pVDZ.json", False),
             ("co_ccpvtz_j", "cc-pVTZ.json", True)]


def part_bse():
    """The reference's data/basis documents (BSE JSON, molssi_bse_schema),
    cut to H, C, N, O, F and their electron shells, values verbatim."""
    out = {}
    for f in BSE_SETS:
        d = json.load(open(os.path.join(REF, "data", "basis", f)))
        out[f] = {"molssi_bse_schema": d["molssi_bse_schema"], "name": d["name"],
                  "function_types": d["function_types"],
                  "elements": {z: {"electron_shells": d["elements"][z]["electron_shells"]}
                               for z in BSE_ELEMENTS}}
    # the reference's own mapping (test/oracle/basis.py from_bse) of these
    # documents onto shells, for the atoms of the one-electron fixtures
    sys.path.insert(0, os.path.join(REF, "test"))
    from felizjueves.ao import bse as ref_bse
    from oracle.basis import from_bse as ref_from_bse
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for case, f, reduce in BSE_CASES:
        d = json.load(open(os.path.join(fx, case + ".json")))
        atoms = [(a["charge"], tuple(a["coord"])) for a in d["atoms"]]
        B = ref_from_bse(ref_bse.load(os.path.join(REF, "data", "basis", f)), atoms, reduce=reduce)
        sh = flat_shells([s_.l for s_ in B.shells], [s_.centre for s_ in B.shells],
                         [s_.exponents for s_ in B.shells], [s_.coefficients for s_ in B.shells])
        np.savez_compressed(os.path.join(HERE, f"bse_{case}{'_reduced' if reduce else ''}.npz"), **sh,
                            source=np.asarray(f"reference test/oracle/basis.py from_bse(data/basis/{f}, "
                                              f"atoms of {case}, reduce={reduce})"))
        print("bse mapped", case)
    sys.path.remove(os.path.join(REF, "test"))
    for m in [m for m in sys.modules if m == "oracle" or m.startswith("oracle.")]:
        del sys.modules[m]  # the reference's test oracle, not this repository's
    with open(os.path.join(HERE, "bse_subset.json"), "w") as fh:
        json.dump({"source": "reference data/basis/{" + ",".join(BSE_SETS) + "} (Basis Set Exchange "
                             "JSON, via FreeBreakfast data/basis), elements " + " ".join(BSE_ELEMENTS),
                   "sets": out}, fh, indent=0)
    print("bse", len(out))


NUMERIC_J = [("j_h2o_sto3g_bse", "h2o_sto3g_j"), ("j_h2o_631g_bse", "h2o_631g_j"),
             ("j_h2o_ccpvdz_bse", "h2o_ccpvdz_j"),
             # grad.rhf.get_jk's vj, 3 x n x n
             ("jx1_h2o_sto3g_bse", "h2o_sto3g_j"), ("jx1_h2o_ccpvdz_bse", "h2o_ccpvdz_j")]


def part_numeric_j():
    """The reference's numerical golden store (test/golden/numeric/): PySCF's
    J over a basis read exactly as the BSE document states it (no
    free-primitive reduction), for the density of the fixture its manifest
    names (checked by that manifest's sha256 of the density)."""
    import hashlib
    nd = os.path.join(REF, "test", "golden", "numeric")
    man = json.load(open(os.path.join(nd, "manifest.json")))["entries"]
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for entry, case in NUMERIC_J:
        m = man[entry]
        assert m["density"]["fixture"] == case and m["provenance"]["cart"] is True
        J = np.load(os.path.join(nd, m["file"]))
        d = json.load(open(os.path.join(fx, case + ".json")))
        n = d["nao"]
        D = np.asarray(d["arrays"]["density"]["values"], np.float64).reshape(n, n)
        assert J.shape[-2:] == D.shape
        assert hashlib.sha256(D.tobytes()).hexdigest() == m["density"]["sha256"]
        np.savez_compressed(os.path.join(HERE, f"numeric_{entry}.npz"), J=J, D=D,
                            basis_file=np.asarray(m["basis"]["file"]),
                            source=np.asarray(f"test/golden/numeric/{m['file']} (PySCF "
                                              f"{m['provenance']['pyscf']}, libcint "
                                              f"{m['provenance']['libcint']}); density of "
                                              f"test/oracle/fixtures/{case}.json"))
        print("numeric", entry, n, hashlib.sha256(D.tobytes()).hexdigest()[:12])


NUMERIC_METRIC = ["metric_h2o_ccpvdz_jkfit_bse", "metric_h2o_def2_universal_jkfit_bse"]


def part_numeric_metric():
    """The numerical golden store's Cartesian (P|Q) over auxiliary BSE
    documents (data/aux_basis/, read as they stand) on the fixtures' H2O,
    with those documents cut to H and O."""
    nd = os.path.join(REF, "test", "golden", "numeric")
    man = json.load(open(os.path.join(nd, "manifest.json")))["entries"]
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for entry in NUMERIC_METRIC:
        m = man[entry]
        assert m["provenance"]["cart"] is True
        V = np.load(os.path.join(nd, m["file"]))
        d = json.load(open(os.path.join(REF, m["basis"]["file"])))
        doc = {"molssi_bse_schema": d["molssi_bse_schema"], "name": d["name"],
               "function_types": d["function_types"],
               "elements": {z: {"electron_shells": d["elements"][z]["electron_shells"]}
                            for z in ("1", "8")}}
        case = m["molecule"]["fixture"]
        atoms = json.load(open(os.path.join(fx, case + ".json")))["atoms"]
        np.savez_compressed(os.path.join(HERE, f"numeric_{entry}.npz"), metric=V,
                            document=np.asarray(json.dumps(doc)),
                            charges=np.asarray([a["charge"] for a in atoms], np.float64),
                            coords=np.asarray([a["coord"] for a in atoms], np.float64),
                            source=np.asarray(f"test/golden/numeric/{m['file']} (PySCF "
                                              f"{m['provenance']['pyscf']}, libcint "
                                              f"{m['provenance']['libcint']}); {m['basis']['file']} "
                                              f"cut to H and O; atoms of test/oracle/fixtures/{case}.json"))
        print("numeric", entry, V.shape)


# --- density fitting: libcint (P|Q) rows and (mn|P) columns -------------------

DF_SETS = {
    "prim_spd_f_auxi_metric": ("metric", "prim_spd_f", ["rows0_56", "rows56_104", "rows104_140",
                                                        "rows140_168"]),
    "h2o_ccpvtz_jkfit_metric": ("metric", "h2o_ccpvdz_j", ["rows0_43", "rows43_81", "rows81_121",
                                                          "rows121_166"]),
    "prim_spd_f_auxi_3c": ("three_center", "prim_spd_f", ["cols0_35", "cols35_84", "cols84_119",
                                                         "cols119_140", "cols140_168"]),
    "h2o_sto3g_jkfit_3c": ("three_center", "h2o_sto3g_j", ["cols0_166"]),
}


def part_df():
    import ast
    fx = os.path.join(REF, "test", "oracle", "fixtures")
    for set_name, (kind, parent, pieces) in DF_SETS.items():
        parts, aux = [], None
        for piece in pieces:
            d = json.load(open(os.path.join(fx, f"{set_name}_{piece}.json")))
            meta = d[kind]
            conv = meta["converted"]
            conv = ast.literal_eval(conv) if isinstance(conv, str) else conv
            if aux is None:
                aux = conv["shells"]
            assert conv["shells"] == aux
            key = [k for k in d["arrays"] if k.startswith("int2c2e_cart" if kind == "metric"
                                                          else "int3c2e_cart")][0]
            a = d["arrays"][key]
            parts.append(np.asarray(a["values"]).reshape(a["shape"]))
        full = np.concatenate(parts, axis=0 if kind == "metric" else 2)
        pj = json.load(open(os.path.join(fx, f"{parent}.json")))
        ao = pj["converted"]["shells"]
        shA = flat_shells([s["l"] for s in ao], [s["centre"] for s in ao],
                          [s["exponents"] for s in ao], [s["coefficients"] for s in ao])
        shX = flat_shells([s["l"] for s in aux], [s["centre"] for s in aux],
                          [s["exponents"] for s in aux], [s["coefficients"] for s in aux])
        np.savez_compressed(os.path.join(HERE, f"df_{set_name}.npz"), value=full, kind=kind,
                            **{"ao_" + k: v for k, v in shA.items()},
                            **{"aux_" + k: v for k, v in shX.items()},
                            source=np.asarray(f"test/oracle/fixtures/{set_name}_*.json"))
        print("df", set_name, full.shape)


# --- Boys -------------------------------------------------------------------


def part_boys():
    _ref_imports()
    from felizjueves.reference.boys import boys
    rng = np.random.default_rng(7)
    T = np.concatenate([
        [0.0, 1e-12, 1e-8, 1e-5, 1e-3, 0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0,
         15.0, 20.0, 25.0, 30.0, 35.0, 36.0, 40.0, 50.0, 75.0, 100.0, 124.9,
         125.0, 150.0, 300.0, 1e3, 1e4, 1e5, 1e6],
        rng.uniform(0, 40, 200), 10 ** rng.uniform(-6, 6, 100)])
    M = np.arange(0, 25)
    F = np.array([[boys(int(m), float(t)) for t in T] for m in M])
    np.savez_compressed(os.path.join(HERE, "boys_ref.npz"), T=T, M=M, F=F)
    print("boys", F.shape)


# --- ERI blocks on sampled quartets -----------------------------------------


def _eri_one(args):
    basis_flat, q = args
    _ref_imports()
    from functools import partial as _p
    from felizjueves.eri.eri import eri_block_and_scale
    from felizjueves.reference.pq import pq
    shells = basis_flat
    a, b, c, d = q
    blk, scale = eri_block_and_scale((shells[a], shells[b]), (shells[c], shells[d]),
                                     pq=pq)
    return (np.asarray(blk, np.float64).ravel(), np.asarray(scale, np.float64).ravel())


def sample_quartets(basis, rng, per_class, max_l_sum=None):
    """Ordered quartets (a,b,c,d) sampled per class (la,lb,lc,ld), shells
    chosen at random among those of each l."""
    by_l = {}
    for i, s in enumerate(basis.shells):
        by_l.setdefault(s.l, []).append(i)
    ls = sorted(by_l)
    out = []
    for la in ls:
        for lb in ls:
            for lc in ls:
                for ld in ls:
                    if max_l_sum is not None and la + lb + lc + ld > max_l_sum:
                        continue
                    for _ in range(per_class):
                        out.append(tuple(int(rng.choice(by_l[x]))
                                         for x in (la, lb, lc, ld)))
    return out


def part_eri():
    _ref_imports()
    from felizjueves_b200 import configs
    rng = np.random.default_rng(11)
    for wname, w, per in (("c0", configs.c0(), 3), ("c1", configs.c1(), 1)):
        rb = ref_basis(w.basis)
        qs = sample_quartets(w.basis, rng, per)
        t = time.time()
        with mp.get_context("spawn").Pool(8) as pool:
            res = pool.map(_eri_one, [(rb.shells, q) for q in qs], chunksize=1)
        vals = np.concatenate([r[0] for r in res])
        scl = np.concatenate([r[1] for r in res])
        offs = np.cumsum([0] + [len(r[0]) for r in res]).astype(np.int64)
        np.savez_compressed(os.path.join(HERE, f"eri_{wname}.npz"),
                            quartets=np.asarray(qs, np.int32), values=vals,
                            scale=scl, offsets=offs)
        print("eri", wname, len(qs), "quartets", round(time.time() - t, 1), "s")


def _eri_pick(args):
    """One quartet's reference block, reduced to a few elements: the one of
    largest |value|, the one of largest scale, and up to `k` more drawn at
    random (seeded by the quartet's position), with the block's largest
    scale."""
    shells, q, k, seed = args
    v, s = _eri_one((shells, q))
    rng = np.random.default_rng(seed)
    pick = [int(np.argmax(np.abs(v))), int(np.argmax(s))]
    if len(v) > 2:
        pick += [int(x) for x in rng.choice(len(v), size=min(k, len(v)), replace=False)]
    pick = sorted(set(pick))
    return pick, v[pick], s[pick], float(s.max())


def part_eri_c1_sample():
    """c1: 40 ordered quartets per class (10,240 in all), each reduced to a
    few elements of the reference's eri_block_and_scale, so the fixture
    stays small."""
    _ref_imports()
    from felizjueves_b200 import configs
    w = configs.c1()
    rb = ref_basis(w.basis)
    rng = np.random.default_rng(12)
    qs = sample_quartets(w.basis, rng, 40)
    t = time.time()
    with mp.get_context("spawn").Pool(8) as pool:
        res = pool.map(_eri_pick, [(rb.shells, q, 6, 1000 + i) for i, q in enumerate(qs)],
                       chunksize=8)
    idx = np.concatenate([np.asarray(r[0], np.int32) for r in res])
    offs = np.cumsum([0] + [len(r[0]) for r in res]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "eri_c1_sample.npz"),
                        quartets=np.asarray(qs, np.int32), offsets=offs, element=idx,
                        values=np.concatenate([r[1] for r in res]),
                        scale=np.concatenate([r[2] for r in res]),
                        block_scale=np.asarray([r[3] for r in res], np.float64))
    print("eri c1 sample", len(qs), "quartets", len(idx), "elements",
          round(time.time() - t, 1), "s")


# --- f_launches plan lists --------------------------------------------------


def _bounds_one(args):
    shells, pairs = args
    _ref_imports()
    from felizjueves.ao.pairs import primitive_schwarz_bounds
    from felizjueves.reference.pq import one_centre
    return [tuple(primitive_schwarz_bounds(shells[a], shells[b],
                                           one_centre=one_centre))
            for a, b in pairs]


def _plan(w, parallel_bounds):
    _ref_imports()
    from felizjueves.ao.pairs import primitive_schwarz_bounds
    from felizjueves.eri.fock.launch_f import f_launches
    from felizjueves.reference.pq import one_centre
    rb = ref_basis(w.basis)
    sh = rb.shells
    t = time.time()
    if parallel_bounds:
        pairs = [(i, j) for i in range(len(sh)) for j in range(i, len(sh))]
        pairs = [(i, j) if (sh[i].l, i) <= (sh[j].l, j) else (j, i) for i, j in pairs]
        chunks = [pairs[k:k + 512] for k in range(0, len(pairs), 512)]
        with mp.get_context("spawn").Pool(8) as pool:
            res = pool.map(_bounds_one, [(sh, c) for c in chunks])
        table = {}
        for c, r in zip(chunks, res):
            for p, g in zip(c, r):
                table[p] = g
        idx = {id(s): i for i, s in enumerate(sh)}

        def bound(sa, sb):
            return table[(idx[id(sa)], idx[id(sb)])]
    else:
        bound = partial(primitive_schwarz_bounds, one_centre=one_centre)
    print("bounds", round(time.time() - t, 1), "s", flush=True)
    P = f_launches(rb, w.D.tolist(), bound=bound, tau=w.tau, n=w.n_mag)
    print("plan", P.counts(), round(time.time() - t, 1), "s", flush=True)
    return P


def save_plan(P, path):
    pairs = P.pairs
    batch_of = []
    for bi, b in enumerate(P.batches):
        batch_of.extend([bi] * len(b.pairs))
    prim_off = np.cumsum([0] + [len(p.prims) for p in pairs]).astype(np.int64)
    np.savez_compressed(
        path,
        tau=P.tau, n=P.n, magnitudes=np.asarray(P.magnitudes), eps=P.eps,
        g_max=P.g_max,
        batch_key=np.asarray([(b.la, b.lb, b.degree, b.mag) for b in P.batches],
                             np.int32),
        batch_npairs=np.asarray([len(b.pairs) for b in P.batches], np.int32),
        pair_ab=np.asarray([(p.a, p.b) for p in pairs], np.int32),
        pair_batch=np.asarray(batch_of, np.int32),
        pair_nprim=np.asarray([p.n_prim for p in pairs], np.int32),
        pair_G=np.asarray([p.G for p in pairs], np.float64),
        pair_dmax=np.asarray([p.dmax for p in pairs], np.float64),
        pair_key=np.asarray([p.key for p in pairs], np.float64),
        pair_mag=np.asarray([p.mag for p in pairs], np.int32),
        prims=np.asarray([k for p in pairs for k in p.prims], np.int32),
        prim_G=np.asarray([g for p in pairs for g in p.prim_G], np.float64),
        prim_off=prim_off,
        launches=np.asarray([(L.bra, L.ket) for L in P.launches], np.int32).reshape(-1, 2),
        screened=np.asarray(P.screened, np.int32).reshape(-1, 2),
        deleted=np.asarray(P.deleted, np.int32).reshape(-1, 2),
        n_prim_total=P.n_prim_total,
        counts=json.dumps(P.counts()))


def part_plan_c0():
    from felizjueves_b200 import configs
    w = configs.c0()
    P = _plan(w, parallel_bounds=False)
    save_plan(P, os.path.join(HERE, "plan_c0.npz"))
    return P


def part_plan_c1():
    from felizjueves_b200 import configs
    w = configs.c1()
    P = _plan(w, parallel_bounds=True)
    save_plan(P, os.path.join(HERE, "plan_c1.npz"))


# --- six-block screen of the c0 plan (walk_f's prediction) -------------------


def part_screen_c0():
    _ref_imports()
    from felizjueves.eri.fock import kernel_f as KF
    from felizjueves_b200 import configs
    w = configs.c0()
    P = _plan(w, parallel_bounds=False)
    rb = ref_basis(w.basis)
    n_sh = len(rb.shells)
    Dsh = KF.density_blocks(w.D.tolist(), rb.offsets, [s.n_cart for s in rb.shells])
    wabs = [abs(KF.WEIGHTS.of(b)) for b in KF.BLOCKS]
    tau = P.tau
    # walk_f.py:344-351, in the kernel's operation order, per launched quartet
    # in the launch's orientation (bra batch's pair first).
    rows = []
    for li, L in enumerate(P.launches):
        diag = L.bra == L.ket
        bras, kets = P.batches[L.bra].pairs, P.batches[L.ket].pairs
        for ib, br in enumerate(bras):
            for ik, kt in enumerate(kets):
                if diag and ik < ib:
                    continue
                s = (br.a, br.b, kt.a, kt.b)
                dmax = wabs[0] * Dsh[s[0] * n_sh + s[1]]
                for wv, (u, v) in zip(wabs[1:], KF.BLOCKS[1:]):
                    t = wv * Dsh[s[u] * n_sh + s[v]]
                    if dmax < t:
                        dmax = t
                skip = br.G * (kt.G * dmax) < tau
                rows.append((li, ib, ik, int(skip)))
    rows = np.asarray(rows, np.int32)
    np.savez_compressed(os.path.join(HERE, "screen_c0.npz"), rows=rows,
                        Dsh=np.asarray(Dsh))
    print("screen_c0", len(rows), "quartets launched,", int(rows[:, 3].sum()), "skipped")


def part_screen_c1():
    """walk_f's six-block prediction (walk_f.py:344-351) on a sample of the
    64-atom cluster's 1.34e9 launched quartets: for every (class, K_AB, K_CD)
    key, the 12 candidates (of 400 drawn) whose bound G_ab (G_cd dmax) lies
    nearest tau -- the decisions a rounding difference would flip -- and 8
    drawn at random.  Rows (launch, ib, ik, skip) in the launch's
    orientation, as screen_c0."""
    _ref_imports()
    from felizjueves.eri.fock import kernel_f as KF
    from felizjueves_b200 import configs
    w = configs.c1()
    P = _plan(w, parallel_bounds=True)
    rb = ref_basis(w.basis)
    n_sh = len(rb.shells)
    t = time.time()
    Dsh = KF.density_blocks(w.D.tolist(), rb.offsets, [s.n_cart for s in rb.shells])
    print("density_blocks", round(time.time() - t, 1), "s", flush=True)
    wabs = [abs(KF.WEIGHTS.of(b)) for b in KF.BLOCKS]
    tau = P.tau

    def bound(br, kt):
        s = (br.a, br.b, kt.a, kt.b)
        dmax = wabs[0] * Dsh[s[0] * n_sh + s[1]]
        for wv, (u, v) in zip(wabs[1:], KF.BLOCKS[1:]):
            x = wv * Dsh[s[u] * n_sh + s[v]]
            if dmax < x:
                dmax = x
        return br.G * (kt.G * dmax)

    by_key = {}
    for li, L in enumerate(P.launches):
        B, K = P.batches[L.bra], P.batches[L.ket]
        diag = L.bra == L.ket
        nq = len(B.pairs) * len(K.pairs) if not diag else \
            len(B.pairs) * (len(B.pairs) + 1) // 2
        by_key.setdefault((B.la, B.lb, K.la, K.lb, B.degree, K.degree), []).append((li, nq))
    rng = np.random.default_rng(11)
    rows = []
    for key in sorted(by_key):
        ls = by_key[key]
        wts = np.asarray([nq for _, nq in ls], np.float64)
        cand = []
        for _ in range(400):
            li = ls[int(rng.choice(len(ls), p=wts / wts.sum()))][0]
            L = P.launches[li]
            bras, kets = P.batches[L.bra].pairs, P.batches[L.ket].pairs
            ib = int(rng.integers(len(bras)))
            ik = int(rng.integers(ib if L.bra == L.ket else 0, len(kets)))
            cand.append((li, ib, ik, bound(bras[ib], kets[ik])))
        cand = list({(c[0], c[1], c[2]): c for c in cand}.values())
        near = sorted(cand, key=lambda c: abs(math.log(max(c[3], 1e-300) / tau)))[:12]
        rest = [c for c in cand if c not in near]
        pick = near + [rest[i] for i in rng.permutation(len(rest))[:8]]
        for li, ib, ik, b in pick:
            rows.append((li, ib, ik, int(b < tau)))
    rows = np.asarray(sorted(rows), np.int32)
    np.savez_compressed(os.path.join(HERE, "screen_c1_sample.npz"), rows=rows,
                        n_launched=np.int64(sum(nq for v in by_key.values() for _, nq in v)))
    print("screen_c1_sample", len(rows), "quartets from", len(by_key), "keys,",
          int(rows[:, 3].sum()), "skipped")


# --- J and K on small nested systems (reference host path) ------------------


def _jk(args):
    which, w = args
    _ref_imports()
    from felizjueves.eri.j_coulomb.j import coulomb_matrix
    from felizjueves.eri.k_exchange.k import exchange_matrix
    from felizjueves.reference.pq import pq
    rb = ref_basis(w.basis)
    t = time.time()
    if which == "J":
        M = coulomb_matrix(rb, w.D.tolist(), pq=pq)
    else:
        M = exchange_matrix(rb, w.D.tolist(), pq=pq)
    return which, np.asarray(M, np.float64), time.time() - t


def _jk_screened(args):
    which, w = args
    _ref_imports()
    from felizjueves.eri.j_coulomb.j import coulomb_matrix
    from felizjueves.eri.k_exchange.k import exchange_matrix
    from felizjueves.reference.pq import pq
    rb = ref_basis(w.basis)
    t = time.time()
    f = coulomb_matrix if which == "J" else exchange_matrix
    M = f(rb, w.D.tolist(), pq=pq, tau=w.tau)
    return which, np.asarray(M, np.float64), time.time() - t


def part_cpu_c0():
    """The reference's own host path on the 6-atom workload at its tau
    (1e-12): coulomb_matrix (j.py:436) and exchange_matrix (k.py:482), each
    single-threaded in its own process, run side by side; G = J - K/2
    (fock.py:106-108).  Records J, K and each one's wall time."""
    from felizjueves_b200 import configs
    w = configs.c0()
    t = time.time()
    with mp.get_context("spawn").Pool(2) as pool:
        res = dict((r[0], r[1:]) for r in pool.map(_jk_screened, [(k, w) for k in ("J", "K")],
                                                     chunksize=1))
    (J, tj), (K, tk) = res["J"], res["K"]
    import platform
    np.savez_compressed(os.path.join(HERE, "cpu_c0.npz"), J=J, K=K, G=J - 0.5 * K, t_J=tj, t_K=tk,
                        tau=w.tau, nproc=os.cpu_count(),
                        cpu=np.asarray(platform.processor() or platform.machine()),
                        source=np.asarray("reference coulomb_matrix + exchange_matrix, pq path, "
                                          "tau 1e-12, one process (one core) each"))
    print("cpu_c0 J", round(tj, 1), "s K", round(tk, 1), "s wall", round(time.time() - t, 1), "s")


def part_jk_small():
    from felizjueves_b200 import configs
    cases = [("c0_1at", configs.sub_workload(configs.c0(), 1)),
             ("c0_2at", configs.sub_workload(configs.c0(), 2)),
             ("c1_1at", configs.sub_workload(configs.c1(), 1))]
    jobs = [(k, w) for _, w in cases for k in ("J", "K")]
    with mp.get_context("spawn").Pool(6) as pool:
        res = pool.map(_jk, jobs, chunksize=1)
    for i, (name, w) in enumerate(cases):
        (_, J, tj), (_, K, tk) = res[2 * i], res[2 * i + 1]
        np.savez_compressed(os.path.join(HERE, f"jk_{name}.npz"), J=J, K=K,
                            D=w.D, t_J=tj, t_K=tk)
        print("jk", name, w.n_ao, "J", round(tj, 1), "s K", round(tk, 1), "s")


# --- the atomic-free scatter's maps (eri/fock/kernel_f_scatter.py) on c0 ----


def part_scatter_c0():
    _ref_imports()
    from felizjueves.eri.fock import kernel_f_scatter as FS
    from felizjueves_b200 import configs
    w = configs.c0()
    P = _plan(w, parallel_bounds=False)
    rb = ref_basis(w.basis)
    off = rb.offsets
    pick, seen = [], set()
    for li, L in enumerate(P.launches):  # each class's first launch, and its first diagonal one
        B, K = P.batches[L.bra], P.batches[L.ket]
        key = (B.la, B.lb, K.la, K.lb, L.bra == L.ket)
        if key not in seen:
            seen.add(key)
            pick.append(li)
    el, ptr, src, meta = [], [], [], []
    for li in pick:
        L = P.launches[li]
        B, K = P.batches[L.bra], P.batches[L.ket]
        bra_ao = [x for p in B.pairs for x in (off[p.a], off[p.b])]
        ket_ao = [x for p in K.pairs for x in (off[p.a], off[p.b])]
        m = FS.scatter_map((B.la, B.lb, K.la, K.lb), len(K.pairs), bra_ao, ket_ao)
        meta.append((li, m.n_el, m.n_slot, len(el) // 2, len(ptr), len(src)))
        el.extend(m.el)
        ptr.extend(m.ptr)
        src.extend(m.src)
    np.savez_compressed(os.path.join(HERE, "scatter_c0.npz"),
                        meta=np.asarray(meta, np.int64), el=np.asarray(el, np.int32),
                        ptr=np.asarray(ptr, np.int32), src=np.asarray(src, np.int32))
    print("scatter_c0", len(pick), "launches,", len(src), "slots")


def part_scatter_c1():
    """The reference's scatter_map on c1 launches, taken from its own c1 plan
    (plan_c1.npz): per (class, diagonal) key the launch with the fewest
    slots, where that is small enough for the reference's pure-Python map.
    Kept as counts and the sha256 of each map's int32 arrays."""
    import hashlib
    _ref_imports()
    from felizjueves.eri.fock import kernel_f_scatter as FS
    from felizjueves_b200 import configs
    w = configs.c1()
    g = np.load(os.path.join(HERE, "plan_c1.npz"))
    off = ref_basis(w.basis).offsets
    key, npairs, ab = g["batch_key"], g["batch_npairs"], g["pair_ab"]
    first = np.concatenate([[0], np.cumsum(npairs)])
    lau = g["launches"]

    def slots(li):
        bi, ki = lau[li]
        la, lb, lc, ld = int(key[bi][0]), int(key[bi][1]), int(key[ki][0]), int(key[ki][1])
        nab = (la + 1) * (la + 2) // 2 * ((lb + 1) * (lb + 2) // 2)
        ncd = (lc + 1) * (lc + 2) // 2 * ((ld + 1) * (ld + 2) // 2)
        return int(npairs[bi]) * int(npairs[ki]) * (nab + ncd)  # a size order, not the layout

    best = {}
    for li, (bi, ki) in enumerate(lau):
        k = (*map(int, key[bi][:2]), *map(int, key[ki][:2]), int(bi == ki))
        if k not in best or slots(li) < slots(best[k]):
            best[k] = li
    pick = sorted(li for li in best.values() if slots(li) < (1 << 16))
    meta, shas = [], []
    for li in pick:
        bi, ki = lau[li]
        la, lb, lc, ld = int(key[bi][0]), int(key[bi][1]), int(key[ki][0]), int(key[ki][1])
        bra_ao = [off[int(x)] for p in ab[first[bi]:first[bi + 1]] for x in p]
        ket_ao = [off[int(x)] for p in ab[first[ki]:first[ki + 1]] for x in p]
        m = FS.scatter_map((la, lb, lc, ld), int(npairs[ki]), bra_ao, ket_ao)
        h = [hashlib.sha256(np.asarray(a, np.int32).tobytes()).hexdigest() for a in (m.el, m.ptr, m.src)]
        meta.append((li, m.n_el, m.n_slot))
        shas.append(h)
        print("  launch", li, m.n_slot, "slots", flush=True)
    np.savez_compressed(os.path.join(HERE, "scatter_c1.npz"), meta=np.asarray(meta, np.int64),
                        sha=np.asarray(shas))
    print("scatter_c1", len(pick), "launches,", sum(x[2] for x in meta), "slots")


# --- the J-engine's launch plan (eri/j_coulomb/launch.py:274-327) on c0 -----


def part_jplan_c0():
    _ref_imports()
    from felizjueves.eri.j_coulomb import j as JJ
    from felizjueves.eri.j_coulomb import launch as JL
    from felizjueves.reference.pq import pq
    from felizjueves_b200 import configs
    w = configs.c0()
    rb = ref_basis(w.basis)
    t = time.time()
    plan = JL.launches(rb, w.D.tolist(), bound=lambda z, L: JJ.pair_bound_pq(z, L, pq=pq),
                       n_batches=1, tau=w.tau)
    bras, kets = {}, {}
    for c in plan:
        bras[c.lp] = c.bras
        kets[c.lq] = c.kets
    out = {"tau": w.tau}
    for L, recs in bras.items():
        out[f"bra{L}_ijp"] = np.array([(r.i, r.j, r.prim) for r in recs], np.int32)
        out[f"bra{L}_G"] = np.array([r.G for r in recs])
    for L, recs in kets.items():
        out[f"ket{L}_ijp"] = np.array([(r.i, r.j, r.prim) for r in recs], np.int32)
        out[f"ket{L}_key"] = np.array([r.key for r in recs])
    np.savez_compressed(os.path.join(HERE, "jplan_c0.npz"), **out)
    print("jplan_c0", sum(len(v) for v in bras.values()), "records,", round(time.time() - t, 1), "s")


def part_jplan_c1():
    """The reference's J-engine launches() on the 64-atom c1 (its bound is a
    function of (zeta, L) alone, so it is memoised; the values are the
    function's own).  The lists are large, so per Hermite order L the file
    keeps the record count, the sha256 of the bra records (i, j, prim) in
    sweep order and of the ket records in sorted order (int32), and every
    64th record's G and key."""
    import functools
    import hashlib
    _ref_imports()
    from felizjueves.eri.j_coulomb import j as JJ
    from felizjueves.eri.j_coulomb import launch as JL
    from felizjueves.reference.pq import pq
    from felizjueves_b200 import configs
    w = configs.c1()
    rb = ref_basis(w.basis)

    @functools.lru_cache(maxsize=None)
    def bound(z, L):
        return JJ.pair_bound_pq(z, L, pq=pq)

    t = time.time()
    plan = JL.launches(rb, w.D.tolist(), bound=bound, n_batches=1, tau=w.tau)
    bras, kets = {}, {}
    for c in plan:
        bras[c.lp] = c.bras
        kets[c.lq] = c.kets
    out = {"tau": w.tau, "stride": 64}
    for L, recs in bras.items():
        ijp = np.array([(r.i, r.j, r.prim) for r in recs], np.int32)
        out[f"bra{L}_n"] = len(recs)
        out[f"bra{L}_sha"] = hashlib.sha256(ijp.tobytes()).hexdigest()
        out[f"bra{L}_G"] = np.array([r.G for r in recs])[::64]
    for L, recs in kets.items():
        ijp = np.array([(r.i, r.j, r.prim) for r in recs], np.int32)
        out[f"ket{L}_sha"] = hashlib.sha256(ijp.tobytes()).hexdigest()
        out[f"ket{L}_key"] = np.array([r.key for r in recs])[::64]
    np.savez_compressed(os.path.join(HERE, "jplan_c1.npz"), **out)
    print("jplan_c1", sum(len(v) for v in bras.values()), "records,", round(time.time() - t, 1), "s")


# --- F_m(0) as the reference's Boys function returns it ---------------------


def part_boys_zero():
    """felizjueves_b200/csrc/boys_zero.h: the reference's F_m(0), m = 0..24
    (its quadrature at T = 0 lands a few ulps from 1/(2m+1)), the table the
    plans' pair bounds read so that they are the reference's to the bit."""
    _ref_imports()
    from felizjueves.reference.boys import boys
    vals = [boys(m, 0.0) for m in range(25)]
    lines = ["// boys_zero.h -- F_m(0), m = 0..24, as the reference's Boys function returns",
             "// them (reference/boys.py:218 _boys: 112-node Gauss-Legendre quadrature at",
             "// T = 0, a few ulps from 1/(2m+1)).  Written by tests/golden/make_golden.py",
             "// part boys_zero.  The plans' primitive Schwarz bounds read these, so the",
             "// bounds, and the orders they decide, are the reference's to the bit.",
             "#pragma once", "", "namespace fjb {", "", "constexpr int kBoysZeroMax = 24;",
             "constexpr double kBoysZero[kBoysZeroMax + 1] = {"]
    lines += [f"    {v.hex()},  // m = {m}" for m, v in enumerate(vals)]
    lines += ["};", "", "}  // namespace fjb", ""]
    with open(os.path.join(REPO, "felizjueves_b200", "csrc", "boys_zero.h"), "w") as f:
        f.write("\n".join(lines))


# --- the split build's ordered pair stream (eri/hjk/launch_hjk.py) ----------


def part_hjk_c0():
    """hjk_launches on c0 in ordered mode, screens "k" and "j" at c0's tau and
    at 1e-6: pairs, batches, launches in full; the visit keys (n_pairs^2
    of them) as a SHA-256 of their float64 bytes in visit order and a
    strided sample; the skipped mask as a SHA-256 of its packed bits and its
    first 2,000 skipped indices."""
    import hashlib
    _ref_imports()
    from felizjueves.ao.pairs import primitive_schwarz_bounds
    from felizjueves.eri.hjk.launch_hjk import hjk_launches
    from felizjueves.reference.pq import one_centre
    from felizjueves_b200 import configs
    w = configs.c0()
    rb = ref_basis(w.basis)
    bound = partial(primitive_schwarz_bounds, one_centre=one_centre)
    out = {}
    t = time.time()
    for screen in ("k", "j"):
        for tau in (w.tau, 1e-6):
            P = hjk_launches(rb, w.D.tolist(), bound=bound, tau=tau, mode="ordered", screen=screen)
            tag = f"{screen}_{'c0tau' if tau == w.tau else '1e-6'}"
            keys = np.array([v.key for v in P.visits], np.float64)
            out[f"{tag}_keys_sha256"] = hashlib.sha256(keys.tobytes()).hexdigest()
            out[f"{tag}_keys_sample"] = keys[::997].copy()
            mask = np.array([v.skipped for v in P.visits], bool)
            out[f"{tag}_skipped_sha256"] = hashlib.sha256(np.packbits(mask).tobytes()).hexdigest()
            out[f"{tag}_skipped_head"] = np.nonzero(mask)[0][:2000].astype(np.int64)
            out[f"{tag}_counts"] = json.dumps(P.counts())
            if screen == "k" and tau == w.tau:
                pairs = P.pairs
                out["pair_ab"] = np.array([(q.a, q.b) for q in pairs], np.int32)
                out["pair_l_deg"] = np.array([(q.la, q.lb, q.degree) for q in pairs], np.int32)
                out["pair_G"] = np.array([q.G for q in pairs], np.float64)
                out["batch_key"] = np.array([(b.la, b.lb, b.degree) for b in P.batches], np.int32)
                out["batch_npairs"] = np.array([len(b.pairs) for b in P.batches], np.int32)
                out["launches"] = np.array([(L.bra, L.ket) for L in P.launches], np.int32)
                out["launch_cls"] = np.array([L.ordered for L in P.launches], np.int32)
            print("hjk", tag, P.counts(), round(time.time() - t, 1), "s", flush=True)
            del P
    out["tau"] = w.tau
    np.savez_compressed(os.path.join(HERE, "hjk_c0.npz"), **out)


# --- the reference's FLOP model (hgp/cost.py) for every class to L=3 ---------


def part_cost():
    _ref_imports()
    from felizjueves.hgp.cost import cost
    from felizjueves.hgp import hrr, vrr
    rows = []
    pc = [(a, b) for a in range(4) for b in range(a, 4)]
    for i, bra in enumerate(pc):
        for ket in pc[i:]:
            for cls in ((*bra, *ket),):
                c = cost(cls)
                v, h = vrr.build(cls), hrr.build(cls)
                rows.append({"class": list(cls), "x": c.x,
                             "y_bra": c.k2["bra"], "y_ket": c.k2["ket"],
                             "z": c.z, "vrr_nodes": v.n_nodes,
                             "boundary": h.n_boundary,
                             "hrr_statements": h.n_statements,
                             "n_eri": h.n_eri,
                             "boys_max_order": c.boys_max_order})
    out = {"source": "reference src/felizjueves/hgp/cost.py:245 cost(cls), "
                     "pruned VRR DAG + bra-first HRR DAG; one + - * / = 1 flop, "
                     "no FMA; Boys/exp/rsqrt named separately",
           "digest_flops_per_eri": 12, "classes": rows}
    path = os.path.join(REPO, "felizjueves_b200", "data", "hgp_cost.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("cost", len(rows), "classes")


PARTS = {"libcint": part_libcint, "eri_libcint": part_eri_libcint, "numeric_j": part_numeric_j,
         "numeric_metric": part_numeric_metric, "df": part_df, "boys": part_boys, "eri": part_eri,
         "eri_c1_sample": part_eri_c1_sample,
         "plan_c0": part_plan_c0, "plan_c1": part_plan_c1,
         "screen_c0": part_screen_c0, "screen_c1": part_screen_c1, "jk_small": part_jk_small,
         "cpu_c0": part_cpu_c0,
         "cost": part_cost, "jplan_c0": part_jplan_c0, "jplan_c1": part_jplan_c1, "scatter_c0": part_scatter_c0, "scatter_c1": part_scatter_c1,
         "onee": part_onee, "scf": part_scf, "bse": part_bse,
         "harmonics": part_harmonics, "grad": part_grad, "rys": part_rys,
         "hjk_c0": part_hjk_c0, "boys_zero": part_boys_zero}
DEFAULT = ["libcint", "eri_libcint", "numeric_j", "numeric_metric", "boys", "cost", "plan_c0", "screen_c0", "eri", "jplan_c0", "scatter_c0"]


def main():
    global REF
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("parts", nargs="*")
    a = ap.parse_args()
    REF = os.path.abspath(a.ref)
    os.environ["FJB_REF"] = REF
    _ref_imports()
    for p in a.parts or DEFAULT:
        t = time.time()
        PARTS[p]()
        print(f"[{p}] {time.time() - t:.1f} s", flush=True)


if __name__ == "__main__":
    main()
