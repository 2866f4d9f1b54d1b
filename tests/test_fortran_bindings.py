"""The Fortran shim fortran/asohf_gpu.f, checked without a Fortran compiler
(none is available here):

* every replaced routine keeps the reference's dummy argument list, name
  for name and in order (tests/golden/reference_dummies.json, written from
  the reference's sources by tests/golden/make_reference_dummies.py, and
  re-read from the sources when they are present);
* every replacement calls the library entry point of its routine;
* the ISO_C_BINDING interfaces name entry points the C header declares,
  with the same number of arguments;
* the BIND(C) derived types list the C structs' fields in the C order;
* the file is valid fixed form: statements in columns 7-72, continuation
  marks in column 6, no tabs.
"""
import json
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "fortran", "asohf_gpu.f")
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_dummies.json")
REFERENCE = "/root/reference"

# replacement -> the entry point (Fortran interface name) it must call
CALLS = {
    "SORT_DM_PARTICLES_LOCALDENSITY": "ASOHF_SORT_LOCALDENSITY",
    "DENSITY": "ASOHF_DENSITY_C",
    "RENORM_DENSITY": "ASOHF_RENORM_C",
    "SORT_DM_PARTICLES_X": "ASOHF_SORT_X_C",
    "PRUNE_POOR_HALOES": "ASOHF_PRUNE_C",
    "CHECK_RUBISH": "ASOHF_CHECK_RUBISH_C",
    "ACCIDENTAL_SUBSTRUCTURE": "ASOHF_ACCIDENTAL_C",
    "HALOFIND_PARTICLES": "ASOHF_HALOFIND_C",
    "OVERLAPPING": "ASOHF_OVERLAPPING_C",
    "SUBSTRUCTURE_PARTICLES": "ASOHF_SUBSTRUCTURE_C",
}


def shim_text():
    return open(SHIM).read()


def joined(src):
    """Fixed-form continuation lines joined; comment lines dropped."""
    out = []
    for ln in src.split("\n"):
        if ln[:1] in ("!", "*", "c", "C") or not ln.strip():
            continue
        if len(ln) > 5 and ln[:5].strip() == "" and ln[5] not in (" ", "0"):
            out[-1] += " " + ln[6:]
        else:
            out.append(ln)
    return out


def program_units(src):
    """{name: body lines} of the top-level SUBROUTINEs after the module."""
    lines = joined(src)
    units, cur = {}, None
    for ln in lines:
        m = re.match(r"\s{6}SUBROUTINE\s+(\w+)\s*\((.*)\)", ln, re.I)
        if m and cur is None:
            cur = m.group(1).upper()
            units[cur] = {"dummies": [a.strip().upper() for a in m.group(2).split(",") if a.strip()],
                          "body": []}
            continue
        if cur is not None:
            if re.match(r"\s*END\s+SUBROUTINE", ln, re.I):
                cur = None
            else:
                units[cur]["body"].append(ln)
    return units


def test_replacements_keep_the_reference_dummy_lists():
    ref = json.load(open(GOLDEN))
    units = program_units(shim_text())
    assert set(ref) <= set(units), sorted(set(ref) - set(units))
    for name, r in ref.items():
        assert units[name]["dummies"] == r["dummies"], name


def test_golden_dummies_match_the_reference_sources():
    if not os.path.isdir(REFERENCE):
        pytest.skip("reference sources not present")
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mkdum", os.path.join(ROOT, "tests", "golden", "make_reference_dummies.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    ref = json.load(open(GOLDEN))
    for name, fn in mk.ROUTINES.items():
        txt = open(os.path.join(REFERENCE, fn), errors="replace").read()
        hits = [a for n, a, _ in mk.subroutine_statements(txt) if n == name]
        assert hits == [ref[name]["dummies"]], name


def test_each_replacement_calls_its_entry_point():
    units = program_units(shim_text())
    for name, fn in CALLS.items():
        body = " ".join(units[name]["body"]).upper()
        assert re.search(r"\b%s\s*\(" % fn, body), f"{name} does not call {fn}"
        assert "ASOHF_CHECK(" in body, f"{name} does not check the status"
    for name in ("HALOFIND_PARTICLES", "SUBSTRUCTURE_PARTICLES"):
        assert "ASOHF_PPH_BACK" in " ".join(units[name]["body"]).upper()


def fortran_bindings():
    lines = joined(shim_text())
    out = {}
    for ln in lines:
        m = re.search(r"FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*BIND\(C,\s*NAME='(\w+)'\)", ln, re.I)
        if m:
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
    assert len(fb) >= 15
    for name, nargs in fb.items():
        assert name in cd, f"{name} is bound in Fortran but not declared in the header"
        assert cd[name] == nargs, f"{name}: {nargs} Fortran arguments, {cd[name]} in C"


def c_struct_fields(name):
    txt = open(os.path.join(ROOT, "include", "asohf_types.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), txt, re.S)
    fields = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"^(const\s+)?\w+\s*", "", decl)
        fields += [f.strip().lstrip("*").strip() for f in decl.split(",")]
    return [f.upper() for f in fields]


def fortran_type_fields(name):
    lines = joined(shim_text())
    fields, inside = [], False
    for ln in lines:
        if re.match(r"\s*TYPE,\s*BIND\(C\)\s*::\s*%s\b" % name, ln, re.I):
            inside = True
            continue
        if inside:
            if re.match(r"\s*END\s+TYPE", ln, re.I):
                break
            decl = ln.split("::", 1)[1]
            for part in decl.split(","):
                fields.append(part.split("=")[0].strip().upper())
    return fields


@pytest.mark.parametrize("fname,cname", [("ASOHF_MESH_T", "asohf_mesh"),
                                         ("ASOHF_PARTICLES_T", "asohf_particles"),
                                         ("ASOHF_CONSTS_T", "asohf_consts"),
                                         ("ASOHF_CATALOGUE_T", "asohf_catalogue")])
def test_bind_c_types_follow_the_c_structs(fname, cname):
    assert fortran_type_fields(fname) == c_struct_fields(cname)


def test_fixed_form_layout():
    for no, ln in enumerate(shim_text().split("\n"), 1):
        assert "\t" not in ln, f"tab on line {no}"
        if ln[:1] in ("!", "*", "c", "C") or not ln.strip():
            continue
        assert len(ln) <= 72, f"line {no} runs past column 72"
        assert ln[:5].strip() == "", f"line {no}: columns 1-5 hold no label here"
        if ln[5] != " ":
            assert ln[5] == "&", f"line {no}: continuation mark other than &"
