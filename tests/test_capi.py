"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point declared in include/ipeps_b200.h (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(ipeps_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_header_symbols(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares exactly the header's entry points
    assert set(pkg.EXPORTED) <= set(syms)


def test_python_binding_covers_header(pkg):
    assert set(declared_symbols()) <= set(pkg.EXPORTED) | {"ipeps_last_error"} | set(
        s for s in declared_symbols() if s.startswith("ipeps_") and s not in pkg.EXPORTED and "noalloc" in s)


def test_missing_library_fails_loudly(tmp_path, pkg):
    from importlib import import_module
    host = import_module("ipeps_b200.host")
    with pytest.raises(ImportError):
        host._lib, saved = None, host._lib
        try:
            host.load_library(str(tmp_path / "nope.so"))
        finally:
            host._lib = saved


def test_package_exports_what_the_gpu_tests_call(pkg):
    """Every ``pkg.<name>`` the GPU tests use exists on the package (checked
    here, without a GPU, so a missing export does not first show on a B200)."""
    import re
    here = os.path.dirname(os.path.abspath(__file__))
    names = set()
    for f in os.listdir(here):
        if f.endswith("_gpu.py") or f == "test_zz_no_alloc.py":
            with open(os.path.join(here, f)) as fh:
                names |= set(re.findall(r"\bpkg\.([A-Za-z_]\w*)", fh.read()))
    missing = sorted(n for n in names if not hasattr(pkg, n))
    assert not missing, missing
