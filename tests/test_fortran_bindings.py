"""The ISO_C_BINDING interfaces of fortran/asohf_gpu_mod.f90 name entry
points the C header declares, with the same number of arguments (the
module cannot be compiled here: no Fortran compiler)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def fortran_bindings():
    src = open(os.path.join(ROOT, "fortran", "asohf_gpu_mod.f90")).read()
    # join fixed-form continuation lines ("     &" in column 6)
    src = re.sub(r"\n\s*&", " ", src)
    out = {}
    for m in re.finditer(r"FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*BIND\(C,\s*NAME='(\w+)'\)", src, re.I):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        out[m.group(3)] = len(args)
    return out


def c_declarations():
    txt = open(os.path.join(ROOT, "include", "asohf_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"(?:int|int64_t|const char \*)\s*\*?\s*(asohf_\w+)\s*\(([^)]*)\)\s*;", txt):
        params = [p for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        out[m.group(1)] = len(params)
    return out


def test_every_binding_matches_the_header():
    fb, cd = fortran_bindings(), c_declarations()
    assert len(fb) >= 12
    for name, nargs in fb.items():
        assert name in cd, f"{name} is bound in Fortran but not declared in the header"
        assert cd[name] == nargs, f"{name}: {nargs} Fortran arguments, {cd[name]} in C"
