"""The C ABI: libfjb.so loads and exports every function include/fjb.h
declares (no compute call needs a GPU here)."""

import ctypes
import os
import re

from conftest import REPO


def declared():
    src = open(os.path.join(REPO, "include", "fjb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fjb_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(lib_built):
    lib = ctypes.CDLL(lib_built)
    names = declared()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(lib_built):
    from felizjueves_b200 import _lib
    assert set(declared()) <= set(_lib.EXPORTS) | {"fjb_class_info"}


def test_version_and_error_without_gpu(lib_built):
    from felizjueves_b200 import _lib
    L = _lib.load()
    assert b"sm_100a" in L.fjb_version()
    h = ctypes.c_void_p()
    rc = L.fjb_create(ctypes.byref(h), None, 0)
    assert rc == -1
    assert b"no basis" in L.fjb_last_error(None)


def test_product_has_no_cpu_path():
    """The product package never imports the oracle."""
    pkg = os.path.join(REPO, "felizjueves_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh")):
                txt = open(os.path.join(root, f)).read()
                assert "oracle." not in txt.replace("the oracle", ""), f
                assert "import oracle" not in txt and "from oracle" not in txt, f
