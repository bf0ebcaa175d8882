"""CPU checks of the drop-in boundary: struct layout and that every declared C symbol is
exported by the built library (nothing is called, so no GPU is needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER_LIB = {
    "ntt.h": "libntt.so",
    "msm.h": "libmsm.so",
    "poly.h": "libpoly.so",
    "zkp_gen.h": "libzkp_gen.so",
    "zkp_runtime.h": "libzkp_runtime.so",
    "zkp_pipeline.h": "libzkp_pipeline.so",
}


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"\btypedef\b[^;]*;", "", text)  # function-pointer and struct typedefs
    return sorted(set(re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", text)) - {"if", "while", "for", "sizeof"})


@pytest.mark.parametrize("header", sorted(HEADER_LIB))
def test_library_exports_every_declared_symbol(zk, header):
    path = os.path.join(ROOT, "zkpoly-compiler_b200", "lib", HEADER_LIB[header])
    if not os.path.exists(path):
        from importlib import import_module
        import_module("zkpoly-compiler_b200.build").build_all()
    lib = ctypes.CDLL(path)
    names = declared_functions(header)
    assert names, header
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_polyptr_layout(zk):
    P = zk.native.PolyPtr
    assert ctypes.sizeof(P) == 40
    assert [f[0] for f in P._fields_] == ["ptr", "len", "rotate", "offset", "whole_len"]
    assert P.len.offset == 8 and P.whole_len.offset == 32


def test_reference_stage_plan_helpers(zk):
    # GenPqOmegas::get_pq_len (core/src/ntt.rs:322-335) for 32-byte fields, caps (8, 8)
    assert zk.ntt.get_pq_len(16) == 1 << 7
    assert zk.ntt.get_pq_len(24) == 1 << 5
