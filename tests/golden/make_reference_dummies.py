"""Writes tests/golden/reference_dummies.json: the dummy-argument lists of
the reference subroutines that fortran/asohf_gpu.f replaces, read from the
reference's sources (fixed-form Fortran, continuation in column 6).

Run where the reference tree is present:
    python tests/golden/make_reference_dummies.py /path/to/ASOHF
"""
import json
import os
import re
import sys

# routine -> reference file that defines it
ROUTINES = {
    "SORT_DM_PARTICLES_LOCALDENSITY": "reader.f",
    "DENSITY": "grids.f",
    "RENORM_DENSITY": "grids.f",
    "SORT_DM_PARTICLES_X": "grids.f",
    "PRUNE_POOR_HALOES": "haloes_particles.f",
    "CHECK_RUBISH": "haloes_particles.f",
    "ACCIDENTAL_SUBSTRUCTURE": "haloes_particles.f",
    "HALOFIND_PARTICLES": "haloes_particles.f",
    "OVERLAPPING": "haloes_grids.f",
    "SUBSTRUCTURE_PARTICLES": "substructure.f",
}


def subroutine_statements(text):
    """(name, [dummies], line) of every SUBROUTINE statement of a fixed-form
    source, continuation lines joined."""
    lines = text.split("\n")
    out = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln[:1] in ("c", "C", "*", "!"):
            i += 1
            continue
        m = re.match(r"\s+subroutine\s+(\w+)\s*(\(.*)?$", ln.split("!")[0], re.I)
        if not m:
            i += 1
            continue
        start = i
        stmt = ln.split("!")[0]
        while i + 1 < len(lines) and len(lines[i + 1]) > 5 and lines[i + 1][:5].strip() == "" \
                and lines[i + 1][5] not in (" ", "0"):
            i += 1
            stmt += lines[i][6:].split("!")[0]
        m = re.match(r"\s*subroutine\s+(\w+)\s*\((.*)\)", stmt, re.I | re.S)
        if m:
            args = [a.strip().upper() for a in m.group(2).split(",") if a.strip()]
            out.append((m.group(1).upper(), args, start + 1))
        i += 1
    return out


def main(root):
    res = {}
    for name, fn in ROUTINES.items():
        txt = open(os.path.join(root, fn), errors="replace").read()
        hits = [(a, ln) for n, a, ln in subroutine_statements(txt) if n == name]
        assert len(hits) == 1, (name, fn, hits)
        res[name] = {"file": fn, "line": hits[0][1], "dummies": hits[0][0]}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_dummies.json")
    with open(out, "w") as f:
        json.dump(res, f, indent=1)
    print(out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
