"""The C-ABI library loads and exports every symbol include/vilma_gpu.h
declares; host-side argument handling works without a GPU (no compute)."""
import ctypes as C
import os
import re

import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200.abi import VgInfo, VgParams

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "vilma_gpu.h")


def declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(vg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "vg_create" in names and "vg_update" in names and "vg_last_error" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    L = vlib.lib()
    for name in declared():
        assert hasattr(L, name), name
    assert set(vlib.EXPORTS) <= set(declared())


def test_struct_layout_matches_header():
    # field counts of the two structs agree with the header (catches drift between header and ctypes)
    txt = open(HDR).read()
    body = txt[txt.index("typedef struct vg_params {"): txt.index("} vg_params;")]
    fields = re.findall(r"\b(?:int|double)\s+([^;]+);", body)
    names = [n.strip().split("[")[0] for f in fields for n in f.split(",")]
    assert names == [f[0] for f in VgParams._fields_]
    body = txt[txt.index("typedef struct vg_info {"): txt.index("} vg_info;")]
    fields = re.findall(r"\b(?:int|double|long long)\s+([^;]+);", body)
    names = [n.strip() for f in fields for n in f.split(",")]
    assert names == [f[0] for f in VgInfo._fields_]


def test_params_default_is_host_only():
    p = vlib.default_params()
    assert p.n_layer == 4 and p.deg1_cm == 1 and p.sle_n_inner == 20 and abs(p.sle_tol - 1e-7) < 1e-20


def test_bad_arguments_return_status_not_abort():
    L = vlib.lib()
    assert L.vg_create(None, None) != 0
    assert b"null" in L.vg_last_error(None)
