"""The C ABI library loads here (no GPU) and exports every declared symbol."""
import ctypes
import os
import re

import pytest

import prandtl_b200
from prandtl_b200 import cases

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(pdg_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("pdg_create", "pdg_rhs", "pdg_rk_stage", "pdg_rk3_step", "pdg_max_char_speed", "pdg_destroy"):
        assert s in syms


@pytest.mark.parametrize("sym", declared_symbols())
def test_library_exports_symbol(sym):
    lib = prandtl_b200.library()
    assert hasattr(lib, sym), f"{sym} declared in include/ but not exported"


def test_default_params_match_reference_defaults():
    p = prandtl_b200.default_params()
    assert p.gamma == 1.4 and p.alpha_max == 0.5 and p.alpha_min == 0.001
    assert p.blending == 1 and p.compat == 1 and p.face_dissipation == 1.0


def test_create_rejects_bad_arguments_without_a_gpu():
    lib = prandtl_b200.library()
    out = ctypes.c_void_p()
    assert lib.pdg_create(None, None, ctypes.byref(out)) == 1
    mesh = cases.vortex_mesh(2, 3)
    m = prandtl_b200.PdgMesh(2, 9, mesh.num_elements, (ctypes.c_double * 3)(1, 1, 1),
                             mesh.nbr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    p = prandtl_b200.default_params()
    assert lib.pdg_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(out)) == 1  # order 9 unsupported
    assert not out.value
