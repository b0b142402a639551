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


def test_integration_ctypes_binding_runs_on_the_host(lib_built):
    """The ctypes binding INTEGRATION.md shows, run as written (its first
    code block) on a host-only handle: the c0 plan goes through with the
    density passed by pointer, the build refuses with the library's message
    (no device on a host-only handle), and an asymmetric density is refused
    as the reference refuses it."""
    import re
    import subprocess
    import sys
    doc = open(os.path.join(REPO, "INTEGRATION.md")).read()
    block = re.findall(r"```python\n(.*?)```", doc, re.S)[0]
    code = block + (
        "\nfrom felizjueves_b200 import configs\n"
        "w = configs.c0()\n"
        "try:\n"
        "    g_build(w.basis, w.D, tau=w.tau, device=-1)\n"
        "except RuntimeError as e:\n"
        "    assert 'host-only' in str(e), e\n"
        "else:\n"
        "    raise AssertionError('a host-only handle built')\n"
        "D = w.D.copy(); D[2, 5] += 1e-3\n"
        "try:\n"
        "    g_build(w.basis, D, device=-1)\n"
        "except ValueError as e:\n"
        "    assert 'not symmetric' in str(e), e\n"
        "else:\n"
        "    raise AssertionError('an asymmetric density was planned')\n"
        "print('BINDING_OK')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=REPO, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "BINDING_OK" in r.stdout, r.stderr[-2000:]
