"""The Julia binding (ipeps.jl_b200/julia/IPEPSB200.jl) cannot run here (no
Julia toolchain), so its calls are checked against the C ABI statically:
every `ccall((:name, lib), ...)` names a function that include/ipeps_b200.h
declares and libipeps_b200.so exports, with as many argument types as the C
declaration has parameters."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "ipeps.jl_b200", "julia", "IPEPSB200.jl")
HDR = os.path.join(ROOT, "include", "ipeps_b200.h")


def _split_top(s):
    """Split on commas outside braces/parentheses; drop empty trailing items."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "{(":
            depth += 1
        elif ch in "})":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _c_decls():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    decls = {}
    for m in re.finditer(r"IPEPS_API\s+[\w\s\*]+?\b(ipeps_\w+)\s*\(([^;]*?)\)\s*;", src, flags=re.S):
        params = m.group(2).strip()
        decls[m.group(1)] = 0 if params in ("", "void") else len(_split_top(params))
    return decls


def _jl_calls():
    src = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*lib\),\s*[\w{}]+,\s*\(", src):
        # the argument-type tuple starts at the "(" just matched; find its end
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(src[i], 0)
            i += 1
        calls.append((m.group(1), len(_split_top(src[m.end():i - 1]))))
    return calls


def test_every_ccall_matches_a_declared_function():
    decls = _c_decls()
    calls = _jl_calls()
    assert len(calls) >= 15, calls
    for name, nargs in calls:
        assert name in decls, f"{name} is not declared in ipeps_b200.h"
        assert nargs == decls[name], f"{name}: {nargs} argument types in the binding, {decls[name]} in the header"


def test_every_ccall_is_exported_by_the_library():
    lib = os.path.join(ROOT, "ipeps.jl_b200", "libipeps_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    import ctypes
    so = ctypes.CDLL(lib)
    for name, _ in _jl_calls():
        assert hasattr(so, name), name
