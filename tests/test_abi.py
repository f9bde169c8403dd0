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


C_PROGRAM = r"""
#include <stddef.h>
#include <stdio.h>
#include "vilma_gpu.h"

int main(void) {
  vg_params p;
  vg_handle* h = NULL;
  if (vg_params_default(&p) != 0) return 2;
  /* sizes and a few offsets for the ctypes mirror */
  printf("%zu %zu %zu %zu %zu\n", sizeof(vg_params), sizeof(vg_info), offsetof(vg_params, toroidal),
         offsetof(vg_params, sle_ctas), offsetof(vg_info, n_launch));
  printf("%d %d\n", p.n_layer, p.deg1_cm);
  /* a null argument is a status and a message, not an abort */
  if (vg_create(NULL, &h) == 0) return 3;
  printf("%s\n", vg_last_error(NULL));
  return 0;
}
"""


def test_header_is_plain_c_and_links(tmp_path):
    """include/vilma_gpu.h compiles as C99 and a C program links against the
    library (the drop-in boundary: no C++ or torch types); the struct sizes
    and offsets a C caller sees are the ctypes mirror's."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi_c.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "abi_c"
    libdir = os.path.dirname(vlib.LIB_PATH)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.dirname(HDR), str(src), "-o", str(exe),
                        "-L", libdir, "-lvilma_gpu", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0, run.stdout + run.stderr
    lines = run.stdout.splitlines()
    sp, si, o_tor, o_ctas, o_launch = map(int, lines[0].split())
    assert sp == C.sizeof(VgParams) and si == C.sizeof(VgInfo)
    assert o_tor == VgParams.toroidal.offset and o_ctas == VgParams.sle_ctas.offset
    assert o_launch == VgInfo.n_launch.offset
    assert lines[1] == "4 1"
    assert "null" in lines[2]


def test_library_exports_nothing_undeclared():
    """Every vg_* symbol the library exports is declared in the header."""
    import shutil
    import subprocess

    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("no nm")
    r = subprocess.run([nm, "-D", "--defined-only", vlib.LIB_PATH], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    exported = {ln.split()[-1] for ln in r.stdout.splitlines() if ln.split() and ln.split()[-1].startswith("vg_")}
    assert exported, "no vg_ symbols exported"
    assert exported <= set(declared()), sorted(exported - set(declared()))


def test_fortran_binding_matches_header():
    """The iso_c_binding module INTEGRATION.md gives a maintainer binds
    header functions by their C names with the C argument count, and every
    header entry point a Fortran host can use is bound."""
    root = os.path.dirname(HDR)
    txt = open(os.path.join(os.path.dirname(root), "INTEGRATION.md")).read()
    mod = txt[txt.index("module vilma_gpu"): txt.index("end module vilma_gpu")]
    hdr = open(HDR).read()
    c_args = {}
    for name, args in re.findall(r"^(?:int|const char\*)\s+(vg_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", hdr, re.M):
        a = args.strip()
        c_args[name] = 0 if a in ("", "void") else a.count(",") + 1
    f_sigs = re.findall(r"function\s+(vg_[a-z0-9_]+)\s*\(([^)]*)\)\s*&?\s*(?:bind\(c,\s*name=\"(vg_[a-z0-9_]+)\"\))?",
                        mod.replace("&\n", " "))
    bound = {}
    for fname, args, cname in f_sigs:
        if fname in ("vg_check",):
            continue
        n = len([x for x in args.replace("&", " ").split(",") if x.strip()])
        bound[cname or fname] = n
    assert bound, "no bound functions found"
    for name, n in bound.items():
        assert name in c_args, name
        assert n == c_args[name], (name, n, c_args[name])
    device_only = {"vg_update_device", "vg_rsl_device", "vg_stream", "vg_sht_analysis_noalloc", "vg_profile_enable",
                   "vg_profile_read"}
    assert set(c_args) - device_only <= set(bound), sorted(set(c_args) - device_only - set(bound))
